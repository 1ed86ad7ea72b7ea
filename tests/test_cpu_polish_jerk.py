"""The jerk-search polishing oracle (max_rzw_arr_harmonics, optimize_accelcand
with numw > 0) against the reference's own battery, tests/test_max_rzw_harmonics.py
of the reference: harmonic signals with average Fourier (r, z, w) drawn as
there (r near N / (4 numharm) plus U(0, 1), z ~ U(-100, 100), w ~ U(-600,
600), injected with its mid-observation parametrisation r0 = r - z/2 + w/12,
z0 = z - w/2), unit-variance noise, starts perturbed by U(-1, 1) x (0.5, 2,
20) / (0.5 numharm).  The reference prints the error statistics; here every
recovered value must lie within one step of the fundamental's search grid
(1/8 bin in r, 1/2 in z, 5 in w) and the power within 5 % of N^2/4.  The
candidates of one spectrum sit 3000 bins apart so that one spectrum carries
them all."""
import os

import numpy as np
import pytest

N = 2 ** 18
THEO_POW = N ** 2.0 / 4.0
# (numharm, fundamental r): every harmonic at least 3000 bins from any other
PLACES = [(3, 3000), (3, 13000), (2, 17000), (2, 22000), (1, 50000), (1, 60000)]


def presto_rfft(sig):
    x = np.fft.rfft(sig)
    out = x[:sig.size // 2].astype(np.complex64)
    out[0] = complex(x[0].real, x[sig.size // 2].real)
    return out


def jerk_spectrum(seed=2024):
    """The spectrum and, per candidate, (numharm, r, z, w, r_start, z_start,
    w_start), drawn as the reference's battery draws them."""
    rng = np.random.default_rng(seed)
    us = np.arange(N, dtype=np.float64) / N
    sig = np.zeros(N)
    cands = []
    for numharm, rbase in PLACES:
        r = rbase + rng.uniform(0.0, 1.0)
        z = rng.uniform(-100, 100)
        w = rng.uniform(-600, 600)
        for ii in range(numharm):
            rh, zh, wh = r * (ii + 1), z * (ii + 1), w * (ii + 1)
            r0 = rh - 0.5 * zh + wh / 12.0
            z0 = zh - 0.5 * wh
            sig += np.cos(2.0 * np.pi * (us * (us * (us * wh / 6.0 + z0 / 2.0) + r0)))
        off = rng.uniform(-1.0, 1.0, 3) * np.array([0.5, 2.0, 20.0]) / (0.5 * numharm)
        cands.append((numharm, r, z, w, r + off[0], z + off[1], w + off[2]))
    sig += rng.standard_normal(N)
    return presto_rfft(sig), cands


@pytest.fixture(scope="module")
def jerk_case():
    return jerk_spectrum()


@pytest.fixture(scope="module")
def jerk_polished(oracle, jerk_case):
    ft, cands = jerk_case
    starts = [(c[0], c[4], c[5], c[6]) for c in cands]
    return oracle.optimize_cands_w(ft, 0, starts, jerk=True, nthreads=os.cpu_count() or 1)


def test_max_rzw_arr_harmonics_recovers_injected_peaks(jerk_case, jerk_polished):
    _, cands = jerk_case
    fails = []
    for c, p in zip(cands, jerk_polished):
        numharm, r, z, w = c[:4]
        dr, dz, dw = p["hirs"][0] - r, p["hizs"][0] - z, p["hiws"][0] - w
        pf = float(np.mean(p["pows"])) / THEO_POW
        if not (abs(dr) <= 0.125 and abs(dz) <= 0.5 and abs(dw) <= 5.0 and 0.95 <= pf <= 1.05):
            fails.append((numharm, dr, dz, dw, pf))
    assert not fails, fails


def test_polished_harmonics_are_exact_multiples(jerk_polished):
    """optimize_accelcand stores harmonic h at h times the fundamental's
    (r, z, w) (src/accel_utils.c:577-581)."""
    for p in jerk_polished:
        h = np.arange(1, len(p["hirs"]) + 1)
        np.testing.assert_allclose(p["hirs"], p["hirs"][0] * h, rtol=1e-15)
        np.testing.assert_allclose(p["hizs"], p["hizs"][0] * h, rtol=1e-15, atol=1e-12)
        np.testing.assert_allclose(p["hiws"], p["hiws"][0] * h, rtol=1e-15, atol=1e-12)
        np.testing.assert_allclose(p["pows"], p["derivs"][:, 0], rtol=0)


def test_rzw_grid_values(jerk_case, jerk_polished):
    """The optimum lies on the highest harmonic's grid: r on 1/8 bin steps
    from that harmonic's lobin, z and w on 1/2 and 5 steps from the scaled
    start (src/maximize_rzw.c:168-174)."""
    _, cands = jerk_case
    for c, p in zip(cands, jerk_polished):
        nh, rs, zs, ws = c[0], c[4], c[5], c[6]
        rtop = p["hirs"][0] * nh
        hhlobin = np.floor(rs * nh) - 1
        assert abs((rtop - hhlobin) * 8 - round((rtop - hhlobin) * 8)) < 1e-6
        kz = (p["hizs"][0] * nh - (zs * nh - 4.0)) / 0.5
        kw = (p["hiws"][0] * nh - (ws * nh - 40.0)) / 5.0
        assert abs(kz - round(kz)) < 1e-6 and 0 <= round(kz) <= 16
        assert abs(kw - round(kw)) < 1e-6 and 0 <= round(kw) <= 16


def test_vol_point_is_corr_complex(oracle):
    """The volume's direct sum equals corr_complex's FFT correlation
    (src/corr_routines.c:5-262): data window from lobin - hw spread to
    numbetween points per bin, the placed response, data x conj(kernel),
    inverse FFT over fftlen, outputs from chopbins = hw numbetween on."""
    rng = np.random.default_rng(5)
    data = (rng.standard_normal(4000) + 1j * rng.standard_normal(4000)).astype(np.complex64)
    nb, z, w = 8, 13.5, -140.0
    hw = oracle.w_resp_halfwidth_acc(z, w)
    numkern = 2 * nb * hw
    resp = oracle.response("w", nb, numkern, z=z, w=w)
    fftlen = 1 << int(np.ceil(np.log2(nb * (2 * hw + 10))))
    numgood = (fftlen - 2 * hw * nb) // nb * nb
    for lobin in (1200, hw // 2):           # the second window starts below bin 0
        begin = lobin - hw
        win = np.zeros(fftlen // nb, np.complex128)
        for i in range(win.size):
            if 0 <= begin + i < data.size:
                win[i] = data[begin + i]
        spread = np.zeros(fftlen, np.complex128)
        spread[::nb] = win
        kern = np.zeros(fftlen, np.complex128)
        kern[:numkern // 2] = resp[numkern // 2:]
        kern[fftlen - numkern // 2:] = resp[:numkern // 2]
        y = np.fft.ifft(np.fft.fft(spread) * np.conj(np.fft.fft(kern)))
        for j in (0, 1, 7, 8, 13, numgood // 2, numgood - 1):
            got = oracle.rzw_vol_point(data, begin, nb, j, resp)
            want = y[hw * nb + j]
            assert abs(got - want) <= 1e-5 * (abs(want) + 1.0), (lobin, j, got, want)


def test_acceleration_branch_unchanged(oracle):
    """With jerk off, optimize_cands_w is the acceleration polishing."""
    us = np.arange(2 ** 14) / 2 ** 14
    r, z = 2 ** 14 / 16.0 + 0.3, 6.0
    sig = sum(np.cos(2 * np.pi * (us * (us * (z * h / 2.0) + (r * h - 0.5 * z * h))))
              for h in (1, 2))
    ft = presto_rfft(sig)
    a = oracle.optimize_cands(ft, 0, [(2, r + 0.1, z - 0.7)])[0]
    b = oracle.optimize_cands_w(ft, 0, [(2, r + 0.1, z - 0.7, 0.0)], jerk=False)[0]
    for k in ("pows", "hirs", "hizs", "derivs"):
        np.testing.assert_array_equal(a[k], b[k])
    assert not np.any(b["hiws"])


def test_max_rzw_arr_single_harmonic(oracle, jerk_case):
    """max_rzw_arr (the -noharmpolish path): a 9 x 9 x 24 grid, z +- 2 and
    w +- 20 around the start; started within half of that from the injected
    (r, z, w) it recovers them within one step (1/8 bin, 0.5, 5)."""
    ft, cands = jerk_case
    rng = np.random.default_rng(77)
    for numharm, r, z, w, *_ in cands:
        if numharm != 1:
            continue
        rs, zs, ws = r + rng.uniform(-0.4, 0.4), z + rng.uniform(-1, 1), w + rng.uniform(-10, 10)
        p, ro, zo, wo, rd = oracle.max_rzw_arr(ft, rs, zs, ws)
        assert abs(ro - r) <= 0.125 and abs(zo - z) <= 0.5 and abs(wo - w) <= 5.0, (ro - r, zo - z, wo - w)
        assert 0.95 <= p / THEO_POW <= 1.05
        # the grid: r from (int) rs - 1 in 1/8 bins, z and w from the start
        assert abs((ro - (int(rs) - 1)) * 8 - round((ro - (int(rs) - 1)) * 8)) < 1e-9
        assert abs((zo - (zs - 2.0)) / 0.5 - round((zo - (zs - 2.0)) / 0.5)) < 1e-9
