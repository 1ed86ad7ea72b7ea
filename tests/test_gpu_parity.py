"""Parity of the CUDA engine (through the C ABI) with the CPU oracle.

Tolerances (FP32 device arithmetic vs the FP64 oracle):
  templates / responses : |dev - orc| <= 2e-6 * max|orc|
  power planes, sums    : |dev - orc| <= 1e-4 * (orc + mean plane power)
  index maps, harmonic adds, hit keys: bit-exact
Candidate lists are compared after excusing threshold crossings whose summed
power lies within 1e-4 relative of the stage's power cut (they may flip
between FP32 and FP64 arithmetic); none occur in these seeded cases.
"""
import json
import os

import numpy as np
import pytest

from presto_b200 import synth

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
DT = 64e-6
PTOL = 1e-4


def _spec(N, seed, pulsars):
    return synth.spectrum(synth.time_series(N, seed, pulsars))


CASES = {
    # standard mode (explicit -wmax 0), 4 harmonics
    "std": dict(N=1 << 17, seed=11, zmax=60, wmax=0, numharm=4,
                pulsars=[dict(r=1500.3, z=12.0, harms=[(0.08, 0.3), (0.05, 1.0), (0.03, 2.0)])]),
    # in-memory mode, 8 harmonics
    "inmem": dict(N=1 << 17, seed=12, zmax=60, wmax=None, numharm=8,
                  pulsars=[dict(r=2222.7, z=-20.0, harms=[(0.06, 0.1)] * 6)]),
    # jerk search
    "jerk": dict(N=1 << 16, seed=13, zmax=20, wmax=40, numharm=2,
                 pulsars=[dict(r=900.2, z=6.0, w=25.0, harms=[(0.12, 0.0), (0.06, 0.5)])]),
    # -locpow (double-tophat local-power normalisation), standard and in-memory
    "std_locpow": dict(N=1 << 17, seed=14, zmax=60, wmax=0, numharm=4, locpow=True,
                       pulsars=[dict(r=1700.6, z=-9.0, harms=[(0.08, 0.2), (0.05, 0.9)])]),
    "inmem_locpow": dict(N=1 << 17, seed=15, zmax=40, wmax=None, numharm=8, locpow=True,
                         pulsars=[dict(r=2048.4, z=14.0, harms=[(0.06, 0.4)] * 5)]),
}


@pytest.fixture(scope="module", params=list(CASES))
def case(request, ablib, oracle):
    c = CASES[request.param]
    fft = _spec(c["N"], c["seed"], c["pulsars"])
    kw = dict(zmax=c["zmax"], wmax=c["wmax"], numharm=c["numharm"], locpow=c.get("locpow", False))
    obs = ablib.obs_init(ablib.make_params(c["N"], DT, fft.size, **kw))
    oobs = oracle.obs_init(oracle.make_params(c["N"], DT, fft.size, **kw))
    assert obs.norm_type == oobs.norm_type == int(kw["locpow"])
    return dict(name=request.param, fft=fft, obs=obs, oobs=oobs, kw=kw, N=c["N"])


def test_response_kats_on_device(ctx):
    k = json.load(open(os.path.join(GOLD, "presto_kats.json")))
    nb, z, w = k["numbetween"], k["z"], k["w"]
    nn = nb * 22 * 2          # max(r, z, w half widths) = 22 bins at z=5, w=40
    pr = np.abs(ctx.gen_response("r", nb, nn)) ** 2
    pz = np.abs(ctx.gen_response("z", nb, nn, z=z)) ** 2
    pw = np.abs(ctx.gen_response("w", nb, nn, z=z, w=w)) ** 2
    assert pr[nn // 2] == k["centre_power_r"]
    assert round(float(pz[nn // 2]) - k["centre_power_z"], k["decimals"]) == 0
    assert round(float(pw[nn // 2]) - k["centre_power_w"], k["decimals"]) == 0


@pytest.mark.parametrize("z,w", [(0.0, 0.0), (2.0, 0.0), (-40.0, 0.0), (200.0, 0.0),
                                 (600.0, 0.0), (10.0, 40.0), (-60.0, 200.0), (100.0, -300.0)])
def test_responses_match_oracle(ctx, oracle, z, w):
    L = oracle.lib(64)
    numkern = 4 * L.orc_w_resp_halfwidth(z, w)
    dev = ctx.gen_response("w", 2, numkern, z=z, w=w)
    orc = oracle.response("w", 2, numkern, z=z, w=w)
    assert np.max(np.abs(dev - orc)) <= 2e-6 * np.max(np.abs(orc))


@pytest.mark.parametrize("kind,nb,z,w", [("r", 2, 0.0, 0.0), ("z", 2, 3.0, 0.0),
                                         ("z", 2, -600.0, 0.0), ("z", 16, 5.0, 0.0),
                                         ("w", 2, 0.0, 40.0), ("w", 16, 5.0, 40.0),
                                         ("w", 2, -60.0, 200.0), ("w", 2, 100.0, -300.0)])
def test_responses_match_reference_build(ctx, oracle, kind, nb, z, w):
    """The device's responses against the reference's own gen_*_response
    (src/responses.c, built unmodified into oracle/_ref when the reference
    tree was present; FFTW stood in for by an FP64 realfft)."""
    ref = oracle.ref_polish_lib()
    if ref is None:
        pytest.skip("no reference build in oracle/_ref")
    numkern = 2 * nb * (32 if kind == "r" else ref.w_resp_halfwidth(z, w, 0))
    want = oracle.ref_response(ref, kind, nb, numkern, z=z, w=w)
    dev = ctx.gen_response(kind, nb, numkern, z=z, w=w)
    assert np.max(np.abs(dev - want)) <= 2e-6 * np.max(np.abs(want))


def test_fundamental_templates_match_oracle(ctx, oracle, ablib, case):
    """Device templates against the oracle's: at the reference's fftlen when
    the device uses it, else the oracle's response placed (centre at index 0,
    place_complex_kernel) and transformed in FP64 at the device length (a
    superblock transform serves several blocks)."""
    obs, oobs = case["obs"], case["oobs"]
    bank = oracle.Bank(oobs, 1, 1)
    hwf = ablib.lib().ab_w_resp_halfwidth
    for wi in sorted({0, bank.nw // 2, bank.nw - 1}):
        for zi in (0, bank.nz // 3, bank.nz - 1):
            dev = ctx.bank_kernel(obs, 1, 1, wi, zi)
            if dev.size == bank.fftlen:
                orc = bank.kernel(wi, zi)
            else:
                z, w = -bank.zmax + 2.0 * zi, -bank.wmax + 20.0 * wi
                numkern = 4 * hwf(z, w)
                resp = oracle.response("w" if w != 0 else "z", 2, numkern, z=z, w=w)
                placed = np.zeros(dev.size, np.complex128)
                half = numkern // 2
                placed[:half] = resp[half:]
                placed[dev.size - half:] = resp[:half]
                orc = np.fft.fft(placed)
            assert np.max(np.abs(dev - orc)) <= 2e-6 * np.max(np.abs(orc)), (wi, zi, dev.size)


def _harmonics(obs):
    hs = [(1, 1)]
    if not obs.inmem:
        for s in range(1, obs.numharmstages):
            hs += [(1 << s, h) for h in range(1, 1 << s, 2)]
    return hs


def _close(dev, orc):
    tol = PTOL * (orc + max(float(orc.mean()), 1e-3))
    return np.all(np.abs(dev - orc) <= tol), float(np.max(np.abs(dev - orc) / (orc + 1.0)))


def test_planes_match_oracle(ctx, oracle, case):
    obs, oobs, fft = case["obs"], case["oobs"], case["fft"]
    ctx.set_spectrum(obs, fft)
    nblk = 0
    startr = obs.rlo
    starts = []
    while startr + obs.rstep < obs.highestbin:
        starts.append(startr)
        startr += obs.rstep
    picks = sorted({0, 1, len(starts) // 2, len(starts) - 1})
    banks = {}
    for (nh, hn) in _harmonics(obs):
        banks[(nh, hn)] = oracle.Bank(oobs, nh, hn)
    for b in picks:
        lo = starts[b]
        hi = lo + obs.rstep - 0.5
        for (nh, hn) in _harmonics(obs):
            meta, dev = ctx.subharm_fderivs_vol(obs, nh, hn, lo, hi)
            ometa, orc, _, _ = oracle.subharm_fderivs_vol(oobs, fft, nh, hn, lo, hi, banks[(nh, hn)])
            assert meta == ometa, (b, nh, hn)
            ok, worst = _close(dev, orc)
            assert ok, (case["name"], b, nh, hn, worst)
            nblk += 1
    assert nblk > 0


def test_add_ffdotpows_bitexact(ctx, oracle, case):
    obs, oobs, fft = case["obs"], case["oobs"], case["fft"]
    if obs.inmem:
        pytest.skip("standard-mode routine")
    ctx.set_spectrum(obs, fft)
    lo = obs.rlo + 3 * obs.rstep
    hi = lo + obs.rstep - 0.5
    fmeta, fund = ctx.subharm_fderivs_vol(obs, 1, 1, lo, hi)
    for (nh, hn) in _harmonics(obs)[1:]:
        smeta, sub = ctx.subharm_fderivs_vol(obs, nh, hn, lo, hi)
        bank = oracle.Bank(oobs, nh, hn)
        _, _, rinds, zinds = oracle.subharm_fderivs_vol(oobs, fft, nh, hn, lo, hi, bank)
        got = ctx.add_ffdotpows(obs, fmeta, fund, smeta, sub, nh, hn, lo)
        f = hn / nh
        exp = fund.copy()
        for ii in range(fmeta["numws"]):
            ww = fmeta["wlo"] + ii * 20
            subw = oracle.lib(64).orc_calc_required_w(f, ww)
            wind = int((subw - smeta["wlo"]) * 0.05 + 1e-14)
            exp[ii] = fund[ii] + sub[wind][zinds[:fmeta["numzs"]]][:, rinds[:fmeta["numrs"]]]
        assert np.array_equal(got.view(np.uint32), exp.view(np.uint32)), (nh, hn)
        fund = got


def test_inmem_add_bitexact(ctx, oracle, case):
    obs = case["obs"]
    if not obs.inmem:
        pytest.skip("in-memory routine")
    rng = np.random.default_rng(5)
    rlen = (obs.highestbin + obs.corr_uselen) * 2
    plane = rng.exponential(1.0, size=(obs.numz, rlen)).astype(np.float32)
    # fill the device plane block by block, as fund_to_ffdotplane does
    step = obs.corr_uselen
    for c0 in range(0, rlen - step + 1, step):
        meta = dict(rlo=c0 // 2, zlo=int(obs.zlo), wlo=0, numrs=step, numzs=obs.numz, numws=1)
        ctx.fund_to_ffdotplane(obs, meta, np.ascontiguousarray(plane[:, c0:c0 + step]))
    filled = (rlen // step) * step
    lo = int(obs.rlo) + 5 * obs.rstep
    meta = dict(rlo=lo, zlo=int(obs.zlo), wlo=0, numrs=obs.corr_uselen, numzs=obs.numz, numws=1)
    fund = np.ascontiguousarray(plane[:, 2 * lo:2 * lo + obs.corr_uselen]).copy()
    for s in range(1, obs.numharmstages):
        for h in range(1, 1 << s, 2):
            f = h / (1 << s)
            got = ctx.inmem_add_ffdotpows(obs, meta, fund, 1 << s, h)
            rinds = ((2 * lo + np.arange(obs.corr_uselen)) * f + 0.5).astype(np.int64)
            assert rinds.max() < filled
            exp = fund.copy()
            for ii in range(obs.numz):
                zz = int(obs.zlo) + 2 * ii
                x = 0.5 * zz * f
                subz = int(x - 0.5 if x < 0 else x + 0.5) * 2
                zind = int((subz - int(obs.zlo)) * 0.5 + 1e-14)
                exp[ii] = fund[ii] + plane[zind][rinds]
            assert np.array_equal(got.view(np.uint32), exp.view(np.uint32)), (s, h)
            fund = got


def _oracle_stage_sums(oracle, case, block):
    obs, oobs, fft = case["obs"], case["oobs"], case["fft"]
    starts, s = [], obs.rlo
    while s + obs.rstep < obs.highestbin:
        starts.append(s)
        s += obs.rstep
    lo, hi = starts[block], starts[block] + obs.rstep - 0.5
    _, fund, _, _ = oracle.subharm_fderivs_vol(oobs, fft, 1, 1, lo, hi, oracle.Bank(oobs, 1, 1))
    sums = [fund.copy()]
    if obs.inmem:
        # the full plane of all blocks up to this one (and the pre-pass)
        rlen = (obs.highestbin + obs.corr_uselen) * 2
        plane = np.zeros((obs.numz, rlen), np.float32)
        fb = oracle.Bank(oobs, 1, 1)
        pre, p = [], 8.0
        while p < obs.rlo:
            pre.append(p)
            p += obs.rstep
        for st in pre + starts[:block + 1]:
            m, pw, _, _ = oracle.subharm_fderivs_vol(oobs, fft, 1, 1, st, st + obs.rstep - 0.5, fb)
            plane[:, 2 * m["rlo"]:2 * m["rlo"] + m["numrs"]] = pw[0]
        rlo = int(lo)
        for st in range(1, obs.numharmstages):
            for h in range(1, 1 << st, 2):
                f = h / (1 << st)
                rinds = ((2 * rlo + np.arange(obs.corr_uselen)) * f + 0.5).astype(np.int64)
                for ii in range(obs.numz):
                    zz = int(obs.zlo) + 2 * ii
                    x = 0.5 * zz * f
                    zind = (int(x - 0.5 if x < 0 else x + 0.5) * 2 - int(obs.zlo)) // 2
                    fund[0, ii] += plane[zind][rinds]
            sums.append(fund.copy())
        return sums
    for st in range(1, obs.numharmstages):
        for h in range(1, 1 << st, 2):
            bank = oracle.Bank(oobs, 1 << st, h)
            m, sub, rinds, zinds = oracle.subharm_fderivs_vol(oobs, fft, 1 << st, h, lo, hi, bank)
            f = h / (1 << st)
            for ii in range(fund.shape[0]):
                subw = oracle.lib(64).orc_calc_required_w(f, -obs.whi + 20 * ii)
                wind = int((subw - m["wlo"]) * 0.05 + 1e-14)
                fund[ii] += sub[wind][zinds[:obs.numz]][:, rinds[:obs.corr_uselen]]
        sums.append(fund.copy())
    return sums


def test_stage_sums_match_oracle(ctx, oracle, case):
    obs, fft = case["obs"], case["fft"]
    starts, s = 0, obs.rlo
    while s + obs.rstep < obs.highestbin:
        starts += 1
        s += obs.rstep
    for block in sorted({1, starts // 2}):
        dev = ctx.block_stage_sums(obs, fft, block)
        orc = _oracle_stage_sums(oracle, case, block)
        for st in range(obs.numharmstages):
            ok, worst = _close(dev[st], orc[st])
            assert ok, (case["name"], block, st, worst)


def _borderline(pw, stage, obs):
    return abs(pw - obs.powcut[stage]) <= 1e-4 * obs.powcut[stage]


def test_search_matches_oracle(ctx, oracle, case):
    obs, fft, kw, N = case["obs"], case["fft"], case["kw"], case["N"]
    dev = ctx.search(obs, fft)
    blk, st, wi, zi, ri, pw = ctx.last_hits()
    ocands, ohits, _ = oracle.accelsearch(oracle.make_params(N, DT, fft.size, **kw), fft,
                                          nthreads=os.cpu_count() or 1)
    dset = {(int(b), int(s), int(w), int(z), int(r)): float(p)
            for b, s, w, z, r, p in zip(blk, st, wi, zi, ri, pw)}
    oset = {(b, s, w, z, r): p for b, s, w, z, r, p in ohits}
    only_d = [k for k in dset if k not in oset and not _borderline(dset[k], k[1], obs)]
    only_o = [k for k in oset if k not in dset and not _borderline(oset[k], k[1], obs)]
    assert not only_d and not only_o, (only_d[:5], only_o[:5])
    assert len(oset) > 0, "seeded case must produce threshold crossings"
    for k in set(dset) & set(oset):
        assert abs(dset[k] - oset[k]) <= PTOL * oset[k], k
    # visit order is the reference's: keys sorted = block, stage, w, z, r
    keys = list(zip(blk, st, wi, zi, ri))
    assert keys == sorted(keys)
    assert len(dev) == len(ocands)
    for d, o in zip(dev, ocands):
        assert d[2] == o[2]
        assert abs(d[3] - o[3]) < 1e-3 and abs(d[4] - o[4]) < 1e-3 and abs(d[5] - o[5]) < 1e-3
        assert abs(d[0] - o[0]) <= PTOL * o[0]
        assert abs(d[1] - o[1]) <= 1e-3 * max(o[1], 1.0)


def test_injected_signal_recovered(ctx, ablib):
    """cfg1 recipe at reduced length: the sinusoid at f=123.4 Hz, z=40 is the
    strongest candidate, within a bin in r and 2 in z."""
    N = 1 << 19
    fft = synth.cfg1_spectrum(N=N, amp=0.05)
    s = ablib.AccelSearch(zmax=200, numharm=8, sigma=2.0, ctx=ctx)
    cands = s(fft, N, DT)
    best = max(cands, key=lambda c: c[1])
    T = N * DT
    assert abs(best[3] * best[2] - 123.4 * T) < 1.0 or abs(best[3] - 123.4 * T) < 1.0
    assert abs(best[4] * best[2] - 40.0) <= 2.0 or abs(best[4] - 40.0) <= 2.0


def test_accelsearch_run_writes_cand_file(ctx, ablib, tmp_path):
    """AccelSearch.run: the search, sort, harmonic removal, polishing and the
    .cand records of src/accelsearch.c:229-284.  The strongest candidate is
    the injected f = 123.4 Hz, z = 40 tone; its record gives that frequency
    through calc_rzwerrs; the file is the raw record array."""
    N = 1 << 19
    fft = synth.cfg1_spectrum(N=N, amp=0.05)
    s = ablib.AccelSearch(zmax=200, numharm=8, sigma=2.0, ctx=ctx)
    path = tmp_path / "cfg1_ACCEL_200.cand"
    res = s.run(fft, N, DT, candfile=str(path))
    cands, pol, props = res["cands"], res["polished"], res["props"]
    assert cands and len(cands) == len(pol) == len(props)
    assert [c[1] for c in cands] == sorted((c[1] for c in cands), reverse=True)
    assert ablib.eliminate_harmonics(ablib.sort_cands(s(fft, N, DT))) == cands
    T = N * DT
    f0 = ablib.calc_rzwerrs(props[0], T).f          # the search's fundamental, r / T
    assert f0 == cands[0][3] / T
    # the tone is harmonic k of the strongest candidate (k = 1 unless a sum won)
    ks = [k for k in range(1, cands[0][2] + 1) if abs(f0 * k - 123.4) < 1.0 / T]
    assert ks, (f0, cands[0])
    # its polished r lies within half a bin of the injected frequency
    assert abs(pol[0]["hirs"][ks[0] - 1] - 123.4 * T) < 0.5
    assert path.stat().st_size == 88 * len(props)
    back = ablib.read_candfile(str(path))
    assert [(p.r, p.z, p.sig) for p in back] == [(p.r, p.z, p.sig) for p in props]


def test_accelsearch_run_writes_reference_files(ctx, ablib, oracle, tmp_path):
    """AccelSearch.run(rootname=...): <root>_ACCEL_<zmax> (text, the .inf
    appended), its .cand and the .txtcand work file (src/accel_utils.c:
    1443-1447, 1667-1685); the text file is the oracle's restatement
    of output_fundamentals + output_harmonics of the same candidates,
    byte for byte."""
    N = 1 << 19
    fft = synth.cfg1_spectrum(N=N, amp=0.05)
    root = str(tmp_path / "cfg1_DM0.00")
    inf = (b" Number of bins in the time series      =  524288     \n"
           b" Width of each time series bin (sec)    =  6.4e-05\n")
    with open(root + ".inf", "wb") as f:
        f.write(inf)
    res = ablib.AccelSearch(zmax=200, numharm=8, sigma=2.0, ctx=ctx).run(fft, N, DT,
                                                                          rootname=root)
    obs = res["obs"]
    assert res["cands"]
    names = ablib.accel_filenames(root, obs)
    assert names["accel"].endswith("cfg1_DM0.00_ACCEL_200")
    assert os.path.getsize(names["cand"]) == 88 * len(res["cands"])
    # .txtcand: one line per candidate an insertion added, in search order; every
    # final candidate was added at some point with its own (numharm, r, z)
    lines = [ln.split() for ln in open(names["txtcand"]).read().splitlines()]
    assert lines and all(len(f) == 7 for f in lines)
    added = {(int(f[2]), float(f[3]), float(f[5])) for f in lines}
    unsorted = ablib.AccelSearch(zmax=200, numharm=8, sigma=2.0, ctx=ctx)(fft, N, DT)
    for c in unsorted:
        assert (c[2], float("%.4f" % c[3]), float("%.4f" % c[4])) in added, c
    got = open(names["accel"], "rb").read()
    want = oracle.accelfile_text(obs.T, float(obs.nph), obs.numw, res["cands"], res["polished"],
                                 inf)
    assert got == want


def test_wrapping_bank_matches_oracle(ctx, ablib, oracle):
    """zmax=100, wmax=200, numharm=16: the reference's 192-point FFT for the
    1/16 harmonic is one sample shorter than the span its valid cells read, so
    its own circular correlation wraps; the device must reproduce that."""
    N = 1 << 16
    fft = _spec(N, 17, [dict(r=600.2, z=5.0, w=30.0, harms=[(0.1, 0.3)] * 4)])
    kw = dict(zmax=100, wmax=200, numharm=16)
    obs = ablib.obs_init(ablib.make_params(N, DT, fft.size, **kw))
    oobs = oracle.obs_init(oracle.make_params(N, DT, fft.size, **kw))
    geo = {(g["numharm"], g["harmnum"]): g for g in ablib.bank_geometry(obs)}
    g = geo[(16, 1)]
    assert 4 * g["hw"] + g["numrs_max"] - 1 > g["fftlen_ref"]      # the wrap is real
    ctx.set_spectrum(obs, fft)
    bank = oracle.Bank(oobs, 16, 1)
    for b in (1, 7, 20):
        lo = obs.rlo + b * obs.rstep
        meta, dev = ctx.subharm_fderivs_vol(obs, 16, 1, lo, lo + obs.rstep - 0.5)
        ometa, orc, _, _ = oracle.subharm_fderivs_vol(oobs, fft, 16, 1, lo, lo + obs.rstep - 0.5, bank)
        assert meta == ometa
        ok, worst = _close(dev, orc)
        assert ok, (b, worst)


def test_search_with_8192_point_transforms(ablib, oracle):
    """A cost table that makes 8192-point superblock transforms cheapest (the
    four-pass FFT, 512-thread CTAs): the search still matches the oracle."""
    c = CASES["std"]
    fft = _spec(c["N"], c["seed"], c["pulsars"])
    kw = dict(zmax=c["zmax"], wmax=c["wmax"], numharm=c["numharm"])
    default = ablib.get_transform_costs()
    table = list(default)
    table[13] = default[12] * 1.5
    ablib.set_transform_costs(table)
    try:
        obs = ablib.obs_init(ablib.make_params(c["N"], DT, fft.size, **kw))
        assert any(b["L"] == 8192 for b in ablib.bank_geometry(obs))
        cx = ablib.Context(0)
        dev = cx.search(obs, fft)
        blk, st, wi, zi, ri, pw = cx.last_hits()
        cx.close()
    finally:
        ablib.set_transform_costs(default)
    ocands, ohits, _ = oracle.accelsearch(oracle.make_params(c["N"], DT, fft.size, **kw), fft,
                                          nthreads=os.cpu_count() or 1)
    dset = {(int(b), int(s), int(w), int(z), int(r)): float(p)
            for b, s, w, z, r, p in zip(blk, st, wi, zi, ri, pw)}
    oset = {(b, s, w, z, r): p for b, s, w, z, r, p in ohits}
    only_d = [k for k in dset if k not in oset and not _borderline(dset[k], k[1], obs)]
    only_o = [k for k in oset if k not in dset and not _borderline(oset[k], k[1], obs)]
    assert not only_d and not only_o, (only_d[:5], only_o[:5])
    for k in set(dset) & set(oset):
        assert abs(dset[k] - oset[k]) <= PTOL * oset[k], k
    assert len(dev) == len(ocands)
