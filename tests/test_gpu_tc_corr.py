"""Parity of the tensor-core correlation paths (AB_CORR_TC_SPLIT_BF16 and
AB_CORR_TC_SPLIT_FP16) with the CPU oracle, at the tolerance of the FP32 FFT
path:

  power planes, sums : |dev - orc| <= 1e-4 * (orc + mean plane power)
  candidates         : the oracle's list, r/z/w within 1e-3 bins, powers
                       within 1e-4 relative

The banded product is evaluated with BF16 hi + lo operands (about 16
significant bits each; the lo.lo product dropped) and FP32 accumulation, so
the expected amplitude error is ~2^-16 of the plane's rms amplitude and the
power error ~2^-15 relative: inside 1e-4 with margin.  FP16 hi + lo parts
carry about 22 significant bits, so that path's error is ~2^-21 relative.
The worst error seen is printed against the FP64 oracle, and the FP16 path's
worst plane error must stay below 2e-5 (four times under the BF16 path's
measured 4.9e-5).
"""
import os

import numpy as np
import pytest

from presto_b200 import synth
from test_gpu_parity import CASES, DT, PTOL, _borderline, _close, _harmonics, _spec

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["bf16", "fp16"])
def tcctx(request, ablib):
    c = ablib.Context(0)
    c.set_corr_path(ablib.CORR_TC_SPLIT_BF16 if request.param == "bf16" else
                    ablib.CORR_TC_SPLIT_FP16)
    c.split = request.param
    yield c
    c.close()


@pytest.fixture(scope="module", params=list(CASES))
def case(request, ablib, oracle):
    c = CASES[request.param]
    fft = _spec(c["N"], c["seed"], c["pulsars"])
    kw = dict(zmax=c["zmax"], wmax=c["wmax"], numharm=c["numharm"], locpow=c.get("locpow", False))
    obs = ablib.obs_init(ablib.make_params(c["N"], DT, fft.size, **kw))
    oobs = oracle.obs_init(oracle.make_params(c["N"], DT, fft.size, **kw))
    return dict(name=request.param, fft=fft, obs=obs, oobs=oobs, kw=kw, N=c["N"])


def _starts(obs):
    out, s = [], obs.rlo
    while s + obs.rstep < obs.highestbin:
        out.append(s)
        s += obs.rstep
    return out


def test_tc_planes_match_oracle(tcctx, oracle, case):
    obs, oobs, fft = case["obs"], case["oobs"], case["fft"]
    tcctx.set_spectrum(obs, fft)
    starts = _starts(obs)
    worst_all = 0.0
    for (nh, hn) in _harmonics(obs):
        bank = oracle.Bank(oobs, nh, hn)
        for b in sorted({0, 1, len(starts) // 2, len(starts) - 1}):
            lo = starts[b]
            meta, dev = tcctx.subharm_fderivs_vol(obs, nh, hn, lo, lo + obs.rstep - 0.5)
            ometa, orc, _, _ = oracle.subharm_fderivs_vol(oobs, fft, nh, hn, lo, lo + obs.rstep - 0.5,
                                                          bank)
            assert meta == ometa, (b, nh, hn)
            ok, worst = _close(dev, orc)
            assert ok, (case["name"], b, nh, hn, worst)
            worst_all = max(worst_all, worst)
    print(f"\n{case['name']} ({tcctx.split}): worst |dev - fp64| / (orc + 1) = {worst_all:.3g}")
    if tcctx.split == "fp16":
        assert worst_all < 2e-5, worst_all


def test_tc_search_matches_oracle(tcctx, oracle, case):
    obs, fft, kw, N = case["obs"], case["fft"], case["kw"], case["N"]
    dev = tcctx.search(obs, fft)
    blk, st, wi, zi, ri, pw = tcctx.last_hits()
    ocands, ohits, _ = oracle.accelsearch(oracle.make_params(N, DT, fft.size, **kw), fft,
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
    for d, o in zip(dev, ocands):
        assert d[2] == o[2]
        assert abs(d[3] - o[3]) < 1e-3 and abs(d[4] - o[4]) < 1e-3 and abs(d[5] - o[5]) < 1e-3
        assert abs(d[0] - o[0]) <= PTOL * o[0]


def test_tc_wrapping_bank_matches_oracle(tcctx, ablib, oracle):
    """The 1/16 bank of zmax=100, wmax=200, numharm=16, whose reference FFT
    wraps into valid cells: the contraction reads the data periodically."""
    N = 1 << 16
    fft = _spec(N, 17, [dict(r=600.2, z=5.0, w=30.0, harms=[(0.1, 0.3)] * 4)])
    kw = dict(zmax=100, wmax=200, numharm=16)
    obs = ablib.obs_init(ablib.make_params(N, DT, fft.size, **kw))
    oobs = oracle.obs_init(oracle.make_params(N, DT, fft.size, **kw))
    tcctx.set_spectrum(obs, fft)
    bank = oracle.Bank(oobs, 16, 1)
    for b in (1, 7, 20):
        lo = obs.rlo + b * obs.rstep
        meta, dev = tcctx.subharm_fderivs_vol(obs, 16, 1, lo, lo + obs.rstep - 0.5)
        ometa, orc, _, _ = oracle.subharm_fderivs_vol(oobs, fft, 16, 1, lo, lo + obs.rstep - 0.5, bank)
        assert meta == ometa
        ok, worst = _close(dev, orc)
        assert ok, (b, worst)


def test_tc_and_fft_paths_agree(tcctx, ctx, ablib):
    """cfg1 recipe at N = 2^19 (in-memory, zmax 200, 8 harmonics): both paths
    give the same candidates."""
    N = 1 << 19
    fft = synth.cfg1_spectrum(N=N, amp=0.05)
    obs = ablib.obs_init(ablib.make_params(N, DT, fft.size, zmax=200, numharm=8))
    a = ctx.search(obs, fft)
    b = tcctx.search(obs, fft)
    assert len(a) == len(b) and len(a) > 0
    for x, y in zip(a, b):
        assert x[2] == y[2]
        assert abs(x[3] - y[3]) < 1e-3 and abs(x[4] - y[4]) < 1e-3
        assert abs(x[0] - y[0]) <= PTOL * x[0]
