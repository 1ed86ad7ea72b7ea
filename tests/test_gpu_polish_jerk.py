"""Device jerk-search polishing (ab_optimize_cands with obs.numw > 0:
max_rzw_arr_harmonics) against the reference's battery and the oracle.

* The battery of the reference's tests/test_max_rzw_harmonics.py (restated
  in test_cpu_polish_jerk.py) through the C ABI: recovered (r, z, w) within
  one grid step of the injected values, power within 5 %.
* Agreement with the oracle: the optimum is a cell of the same (r, z, w)
  grid, so it must be the same cell.  Responses are FP64 transforms rounded
  to float on both sides (the device's phase-split FFTs and the oracle's one
  long FFT agree to ~1e-15 before rounding) and the volume sums are FP64 on
  both sides.  The rzw_interp points of the final derivatives accumulate in
  float in the oracle (as the reference) and in FP64 on the device: powers
  and local powers within 1e-4 relative, phases within 1e-4 rad, first power
  derivatives within 1e-3 of the power per bin.
* Candidates of a real jerk search (N = 2^18, zmax 40, wmax 100, numharm 2):
  the same agreement.
"""
import os

import numpy as np
import pytest

from test_cpu_polish_jerk import N, THEO_POW, jerk_spectrum

pytestmark = pytest.mark.gpu
DT = 64e-6


def _obs(ablib, numbins, zmax=100, wmax=300, numharm=4):
    return ablib.obs_init(ablib.make_params(N, DT, numbins, zmax=zmax, wmax=wmax, numharm=numharm))


def _agree(dev, orc, tag):
    for k, (d, o) in enumerate(zip(dev, orc)):
        info = (tag, k, d["hirs"][0], o["hirs"][0], d["hizs"][0], o["hizs"][0], d["hiws"][0],
                o["hiws"][0])
        np.testing.assert_array_equal(d["hirs"], o["hirs"], err_msg=str(info))
        np.testing.assert_array_equal(d["hizs"], o["hizs"], err_msg=str(info))
        np.testing.assert_array_equal(d["hiws"], o["hiws"], err_msg=str(info))
        dd, od = d["derivs"], o["derivs"]
        assert np.allclose(dd[:, 0], od[:, 0], rtol=1e-4, atol=1e-9 * THEO_POW), info
        assert np.allclose(dd[:, 6], od[:, 6], rtol=1e-4), info
        dphase = np.angle(np.exp(1j * (dd[:, 1] - od[:, 1])))
        assert np.all(np.abs(dphase) <= 1e-4), info
        assert np.all(np.abs(dd[:, 2] - od[:, 2]) <= 1e-3 * np.abs(od[:, 0]) + 1e-6 * THEO_POW), info
        np.testing.assert_array_equal(d["pows"], dd[:, 0])


@pytest.fixture(scope="module")
def jerk_case():
    return jerk_spectrum()


@pytest.fixture(scope="module")
def jerk_oracle(oracle, jerk_case):
    ft, cands = jerk_case
    starts = [(c[0], c[4], c[5], c[6]) for c in cands]
    return oracle.optimize_cands_w(ft, 0, starts, jerk=True, nthreads=os.cpu_count() or 1)


def test_device_rzw_battery(ctx, ablib, jerk_case, jerk_oracle):
    ft, cands = jerk_case
    obs = _obs(ablib, ft.size)
    assert obs.numw > 0 and obs.lobin == 0
    dev = ctx.optimize_cands(obs, ft, [(0.0, 0.0, c[0], c[4], c[5], c[6]) for c in cands])
    _agree(dev, jerk_oracle, "battery")
    fails = []
    for c, d in zip(cands, dev):
        numharm, r, z, w = c[:4]
        dr, dz, dw = d["hirs"][0] - r, d["hizs"][0] - z, d["hiws"][0] - w
        pf = float(np.mean(d["pows"])) / THEO_POW
        if not (abs(dr) <= 0.125 and abs(dz) <= 0.5 and abs(dw) <= 5.0 and 0.95 <= pf <= 1.05):
            fails.append((numharm, dr, dz, dw, pf))
    assert not fails, fails


def test_device_rzw_device_spectrum(ctx, ablib, jerk_case, jerk_oracle):
    """The same through a spectrum already in device memory."""
    import torch
    ft, cands = jerk_case
    obs = _obs(ablib, ft.size)
    dft = torch.from_numpy(ft.view(np.float32).copy()).cuda()
    dev = ctx.optimize_cands(obs, None, [(0.0, 0.0, c[0], c[4], c[5], c[6]) for c in cands],
                             device_ptr=dft.data_ptr())
    _agree(dev, jerk_oracle, "device spectrum")


def test_device_rzw_edges(ctx, ablib, oracle):
    """Candidates near the ends of the spectrum (data outside it read as 0,
    local-power windows clipped) and at w near 0 (z responses)."""
    rng = np.random.default_rng(9)
    n = 1 << 14
    ft = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    obs = _obs(ablib, n)
    starts = [(1, 3.3, 2.0, 0.0), (2, 12.6, -5.0, 30.0), (1, n - 20.2, 4.0, -20.0),
              (3, 40.1, 0.0, 1e-5), (1, 700.45, -0.5, 4.0)]
    dev = ctx.optimize_cands(obs, ft, [(0.0, 0.0, s[0], s[1], s[2], s[3]) for s in starts])
    orc = oracle.optimize_cands_w(ft, 0, starts, jerk=True, nthreads=os.cpu_count() or 1)
    _agree(dev, orc, "edges")


def test_device_rzw_search_candidates(ctx, ablib, oracle):
    """Candidates of a real jerk search, polished on the device and by the
    oracle."""
    from presto_b200 import synth
    n = 1 << 18
    x = synth.time_series(n, 4242, pulsars=[dict(r=5062.3, z=11.0, w=35.0,
                                                 harms=[(0.06, 0.3), (0.04, 1.1)])])
    ft = synth.spectrum(x)
    obs = ablib.obs_init(ablib.make_params(n, DT, ft.size, zmax=40, wmax=100, numharm=2))
    cands = ctx.search(obs, ft)
    assert cands, "the injected pulsar is found"
    top = sorted(cands, key=lambda c: -c[1])[:4]
    dev = ctx.optimize_cands(obs, ft, top)
    orc = oracle.optimize_cands_w(ft, obs.lobin, [(c[2], c[3], c[4], c[5]) for c in top], jerk=True,
                                  nthreads=os.cpu_count() or 1)
    _agree(dev, orc, "search")


def test_device_noharmpolish_jerk(ctx, ablib, oracle, jerk_case):
    """-noharmpolish: max_rzw_arr for every harmonic on its own
    (src/accel_utils.c:585-597), device against the oracle: the same grid
    cell, the volume's maximum power as the harmonic's power, derivatives
    with the starting point's local power."""
    ft, cands = jerk_case
    obs = ablib.obs_init(ablib.make_params(N, DT, ft.size, zmax=100, wmax=300, numharm=4,
                                           noharmpolish=True))
    assert obs.noharmpolish == 1
    sel = [c for c in cands if c[0] <= 2]
    dev = ctx.optimize_cands(obs, ft, [(0.0, 0.0, c[0], c[4], c[5], c[6]) for c in sel])
    for c, d in zip(sel, dev):
        for ii in range(c[0]):
            n = ii + 1
            p, ro, zo, wo, rd = oracle.max_rzw_arr(ft, c[4] * n, c[5] * n, c[6] * n)
            assert (d["hirs"][ii], d["hizs"][ii], d["hiws"][ii]) == (ro, zo, wo), (c, ii)
            assert abs(d["pows"][ii] - p) <= 1e-5 * p
            dd = d["derivs"][ii]
            assert abs(dd[0] - rd.pow) <= 1e-4 * rd.pow
            assert abs(dd[6] - rd.locpow) <= 1e-4 * rd.locpow
