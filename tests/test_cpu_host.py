"""Host-side logic of libaccel_b200.so that needs no GPU: the library loads
and exports every symbol of include/accel_b200.h, create_accelobs geometry
and thresholds, statistics, and the candidate list."""
import os
import re

import numpy as np
import pytest
import scipy.special as sp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_exports_every_declared_symbol(ablib):
    hdr = open(os.path.join(ROOT, "include", "accel_b200.h")).read()
    declared = set(re.findall(r"\b(ab_[a-z0-9_]+)\s*\(", hdr))
    assert declared == set(ablib.accel.EXPORTS)
    L = ablib.lib()
    for name in declared:
        assert hasattr(L, name), name


CONFIGS = [
    dict(N=1 << 20, zmax=200, numharm=8),
    dict(N=1 << 23, zmax=600, numharm=16),
    dict(N=1 << 22, zmax=200, wmax=300, numharm=8),
    dict(N=1 << 21, zmax=50, numharm=8),
    dict(N=1 << 17, zmax=0, numharm=4),
    dict(N=1 << 17, zmax=0, numharm=1, wmax=0),
    dict(N=1 << 18, zmax=37, numharm=32, sigma=3.0),
    dict(N=1 << 19, zmax=100, wmax=45, numharm=2, sigma=5.0),
    dict(N=1 << 19, zmax=100, numharm=4, rlo=100.0, rhi=80000.0),
]


@pytest.mark.parametrize("cfg", CONFIGS)
def test_obs_init_matches_oracle(ablib, oracle, cfg):
    cfg = dict(cfg)
    N = cfg.pop("N")
    p = ablib.make_params(N, 64e-6, N // 2, **cfg)
    o = ablib.obs_init(p)
    q = oracle.obs_init(oracle.make_params(N, 64e-6, N // 2, **cfg))
    for name, _ in ablib.accel.Obs._fields_:
        a, b = getattr(o, name), getattr(q, name)
        if name in ("powcut", "numindep"):
            assert list(a)[:o.numharmstages] == list(b)[:q.numharmstages], name
        else:
            assert a == b, (name, a, b)


def test_statistics_vs_scipy(ablib):
    for numsum in [1, 2, 4, 8, 16, 32]:
        dof = 2 * numsum
        for chi2 in [1.0, 30.0, 90.0, 500.0]:
            lp = ablib.lib().ab_chi2_logp(chi2, dof)
            if chi2 > 1200.0 or (dof > 30 and chi2 > 100.0):
                continue      # the reference's asymptotic branch
            assert abs(lp - np.log(sp.chdtrc(dof, chi2))) < 1e-12 * max(1.0, abs(lp))
        for q in [1e-9, 1e-12, 1e-40]:
            c = 2.0 * ablib.power_for_sigma(-sp.ndtri(q * 1e7), numsum, 1e7)
            assert abs(c - sp.chdtri(dof, q)) < 1e-9 * c


def test_candidate_sigma_matches_oracle(ablib, oracle):
    L = oracle.lib(64)
    rng = np.random.default_rng(3)
    for numsum in [1, 2, 4, 8, 16, 32]:
        for pw in rng.uniform(5, 2000, 40):
            a = ablib.candidate_sigma(pw, numsum, 2.5e7)
            b = L.orc_candidate_sigma(pw, numsum, 2.5e7)
            assert np.float32(a) == np.float32(b) or abs(a - b) < 1e-12 * b


def test_candlist_matches_oracle(ablib, oracle):
    """insert_new_accelcand replayed on random hit streams."""
    L = oracle.lib(64)
    rng = np.random.default_rng(11)
    for trial in range(20):
        mine = ablib.CandList()
        ref = L.orc_list_new()
        for _ in range(400):
            r = float(np.round(rng.uniform(0, 400) * 2) / 2)
            if rng.random() < 0.1:
                r = float(rng.choice([15.0, 30.0, 45.0]))
            p = float(rng.uniform(20, 60))
            s = float(np.float32(rng.uniform(2, 9)))
            a = mine.insert(p, s, 1, r, 2.0, 0.0)
            b = L.orc_list_insert(ref, p, s, 1, r, 2.0, 0.0)
            assert a == b
        n = L.orc_list_get(ref, None, 0)
        arr = (oracle.Cand * n)()
        L.orc_list_get(ref, arr, n)
        L.orc_list_free(ref)
        got = mine.get()
        assert [(c.power, c.sigma, c.r) for c in arr] == [(g[0], g[1], g[3]) for g in got]


def test_sort_and_eliminate(ablib):
    c = [(10.0, 3.0, 1, 100.0, 0, 0), (12.0, 5.0, 2, 200.0, 0, 0), (11.0, 5.0, 1, 50.0, 0, 0),
         (9.0, 4.0, 1, 300.5, 0, 0), (30.0, 9.0, 4, 150.2, 0, 0)]
    s = ablib.sort_cands(c)
    assert [x[3] for x in s] == [150.2, 200.0, 50.0, 300.5, 100.0]
    e = ablib.eliminate_harmonics(s)
    # 300.5 ~ 2*150.2, 50.0 ~ 150.2/3, 100 ~ 150.2*2/3, 200 ~ 150.2*4/3 are removed
    assert [x[3] for x in e] == [150.2]


def test_transform_cost_table_drives_schedule(ablib):
    """The process-wide cost table chooses transform lengths and superblock
    heights; lengths without a measured cost are not used, and every choice
    keeps 4 hw0 + numrs - 1 <= L (the span of one block)."""
    obs = ablib.obs_init(ablib.make_params(1 << 17, 64e-6, 1 << 16, zmax=60, wmax=0, numharm=4))
    default = ablib.get_transform_costs()
    try:
        assert default[13] <= 0.0 and all(default[i] > 0.0 for i in range(9, 13))
        for b in ablib.bank_geometry(obs):
            assert b["L"] <= 4096 and 1 <= b["sbm"] <= 8
            assert 4 * b["hw"] + b["numrs_max"] - 1 <= b["L"]
        cheap8k = list(default)
        cheap8k[13] = default[12] * 1.5
        ablib.set_transform_costs(cheap8k)
        geo = ablib.bank_geometry(obs)
        assert any(b["L"] == 8192 and b["sbm"] > 1 for b in geo)
        ablib.set_transform_costs([0.0] * 16)             # unmeasured: L log2 L up to 4096
        assert all(b["L"] <= 4096 for b in ablib.bank_geometry(obs))
    finally:
        ablib.set_transform_costs(default)
    assert ablib.get_transform_costs() == default


def test_fourier_amplitudes_and_copy(ablib):
    """get_fourier_amplitudes zero-pads past both ends of the spectrum;
    copy_ffdotpows copies geometry and powers (host-only entry points)."""
    import ctypes as C
    obs = ablib.obs_init(ablib.make_params(1 << 12, 64e-6, 1 << 11, zmax=10, numharm=2))
    rng = np.random.default_rng(5)
    fft = (rng.standard_normal(obs.numbins) + 1j * rng.standard_normal(obs.numbins)).astype(np.complex64)
    out = ablib.get_fourier_amplitudes(obs, fft, obs.lobin - 5, 20)
    assert np.all(out[:5] == 0) and np.array_equal(out[5:], fft[:15])
    out = ablib.get_fourier_amplitudes(obs, fft, obs.lobin + obs.numbins - 4, 10)
    assert np.array_equal(out[:4], fft[-4:]) and np.all(out[4:] == 0)
    src_pw = rng.random(2 * 3 * 7).astype(np.float32)
    dst_pw = np.zeros(64, np.float32)
    F = ablib.accel.FFDotPows
    src = F(11, -4, 0, 7, 3, 2, src_pw.ctypes.data_as(C.POINTER(C.c_float)), src_pw.size)
    dst = F(0, 0, 0, 0, 0, 0, dst_pw.ctypes.data_as(C.POINTER(C.c_float)), dst_pw.size)
    assert ablib.lib().ab_copy_ffdotpows(C.byref(src), C.byref(dst)) == 0
    assert (dst.rlo, dst.zlo, dst.numrs, dst.numzs, dst.numws) == (11, -4, 7, 3, 2)
    assert np.array_equal(dst_pw[:src_pw.size], src_pw)
    small = F(0, 0, 0, 0, 0, 0, dst_pw.ctypes.data_as(C.POINTER(C.c_float)), 5)
    assert ablib.lib().ab_copy_ffdotpows(C.byref(src), C.byref(small)) == -4


@pytest.mark.parametrize("bad", [dict(numharm=3), dict(numharm=64), dict(zmax=-2), dict(N=0),
                                 dict(lobin=1 << 20), dict(wmax=-20)])
def test_obs_init_rejects_bad_options(ablib, bad):
    """The reference exits on these (src/accel_utils.c:1467-1487, clig ranges); the
    C ABI returns AB_ERR_ARG and the Python mirror raises."""
    kw = dict(N=1 << 18, zmax=50, numharm=8)
    kw.update(bad)
    N = kw.pop("N")
    with pytest.raises(ablib.AccelError):
        ablib.obs_init(ablib.make_params(N, 64e-6, max(N // 2, 1), **kw))


def test_candlist_worklog_lines_for_added_candidates_only():
    """search_ffdotpows writes a .txtcand line only when insert_new_accelcand
    adds or replaces (src/accel_utils.c:1443-1447): "%-7.2f  %-7.4f  %-2d
    %-14.4f  %-14.9f  %-10.4f %-10.4f" of power, sigma, numharm, r, r/T, z, w."""
    import presto_b200 as pb
    T = 67.108864
    lst = pb.CandList()
    lst.set_worklog(True, T)
    assert lst.insert(30.0, 5.0, 1, 1000.0, 2.0, 0.0) == 1      # new
    assert lst.insert(20.0, 4.0, 2, 1005.0, 4.0, 0.0) == 0      # weaker, within 15 bins
    assert lst.insert(40.0, 6.5, 2, 1007.5, -6.0, 20.0) == 1    # stronger: replaces
    assert lst.insert(12.0, 2.5, 4, 3000.25, 1.5, 0.0) == 1     # new, far away
    lines = lst.worklog().splitlines()
    want = ["%-7.2f  %-7.4f  %-2d  %-14.4f  %-14.9f  %-10.4f %-10.4f" % a for a in (
        (30.0, 5.0, 1, 1000.0, 1000.0 / T, 2.0, 0.0),
        (40.0, 6.5, 2, 1007.5, 1007.5 / T, -6.0, 20.0),
        (12.0, 2.5, 4, 3000.25, 3000.25 / T, 1.5, 0.0))]
    assert lines == want
    assert [c[3] for c in lst.get()] == [1007.5, 3000.25]
    with pytest.raises(pb.AccelError):
        lst.set_worklog(True, 0.0)
