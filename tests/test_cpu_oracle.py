"""Pins of the CPU oracle: the reference's own known-answer tests, the
reference's fresnl.c (golden table), scipy for the GSL-boundary statistics,
and geometry identities of create_accelobs / init_subharminfo."""
import json
import os

import numpy as np
import pytest
import scipy.special as sp

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_response_kats(oracle):
    k = json.load(open(os.path.join(GOLD, "presto_kats.json")))
    L = oracle.lib(64)
    nb, z, w = k["numbetween"], k["z"], k["w"]
    bps = max(16, L.orc_z_resp_halfwidth(z), L.orc_w_resp_halfwidth(z, w))
    nn = nb * bps * 2
    pr = np.abs(oracle.response("r", nb, nn)) ** 2
    pz = np.abs(oracle.response("z", nb, nn, z=z)) ** 2
    pw = np.abs(oracle.response("w", nb, nn, z=z, w=w)) ** 2
    assert pr[nn // 2] == k["centre_power_r"]
    assert round(float(pz[nn // 2]) - k["centre_power_z"], k["decimals"]) == 0
    assert round(float(pw[nn // 2]) - k["centre_power_w"], k["decimals"]) == 0


def test_fresnel_vs_reference_fresnl(oracle):
    g = np.load(os.path.join(GOLD, "fresnel_ref.npz"))
    for x, S, C in zip(g["x"], g["S"], g["C"]):
        s, c = oracle.fresnel(x)
        assert abs(s - S) < 5e-13 and abs(c - C) < 5e-13, (x, s, S, c, C)
    # scipy's fresnel is an independent check of the same integrals
    s2, c2 = sp.fresnel(g["x"])
    assert np.max(np.abs(s2 - g["S"])) < 1e-12 and np.max(np.abs(c2 - g["C"])) < 1e-12


@pytest.mark.parametrize("dof", [2, 4, 8, 16, 32, 64])
def test_chisq_vs_scipy(oracle, dof):
    L = oracle.lib(64)
    for chi2 in [0.5, 3.0, 20.0, 80.0, 300.0, 1100.0]:
        a, b = L.orc_chisq_q(chi2, dof), sp.chdtrc(dof, chi2)
        assert abs(a - b) <= 1e-12 * b + 1e-300
    for q in [0.3, 1e-3, 1e-10, 7.5e-10, 1e-30, 1e-100]:
        a, b = L.orc_chisq_qinv(q, dof), sp.chdtri(dof, q)
        assert abs(a - b) <= 1e-12 * b


def test_gauss_qinv_vs_scipy(oracle):
    L = oracle.lib(64)
    for q in [0.49, 0.1, 1e-5, 1e-20, 1e-100, 1e-250]:
        assert abs(L.orc_gauss_qinv(q) + sp.ndtri(q)) < 1e-12 * abs(sp.ndtri(q))


def test_candidate_sigma_consistency(oracle):
    """power_for_sigma and candidate_sigma are inverses (src/characteristics.c:526-559)."""
    L = oracle.lib(64)
    for numsum in [1, 2, 4, 8, 16, 32]:
        for sig in [2.0, 5.0, 10.0]:
            p = L.orc_power_for_sigma(sig, numsum, 3.0e7)
            assert abs(L.orc_candidate_sigma(p, numsum, 3.0e7) - sig) < 1e-9


def test_geometry_table(oracle):
    """Block geometry of the workload configs (create_accelobs)."""
    cases = [((1 << 20, 200, None, 8), (2048, 1544, 504, 1)),
             ((1 << 23, 600, None, 16), (4096, 2712, 1384, 0)),
             ((1 << 22, 200, 300, 8), (2048, 1436, 612, 0))]
    for (N, zmax, wmax, nh), (fftlen, cu, mk, inmem) in cases:
        o = oracle.obs_init(oracle.make_params(N, 64e-6, N // 2, zmax=zmax, wmax=wmax, numharm=nh))
        assert (o.fftlen, o.corr_uselen, o.maxkernlen, o.inmem) == (fftlen, cu, mk, inmem)


def test_median_even_odd(oracle):
    L = oracle.lib(64)
    a = np.array([5, 1, 4, 2, 3, 9], np.float32)
    assert L.orc_median(a.ctypes.data, 6) == np.float32(3.5)
    assert L.orc_median(a.ctypes.data, 5) == np.float32(3.0)


def test_fft_roundtrip(oracle):
    """FFT round trip (tests/test_presto_python.py:9-29 analogue), mixed radix."""
    L = oracle.lib(64)
    rng = np.random.default_rng(0)
    for n in [20, 384, 1280, 2048]:
        x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex128)
        y = x.copy()
        L.orc_cfft_double.argtypes = [oracle.C.c_void_p, oracle.C.c_int, oracle.C.c_int]
        L.orc_cfft_double(y.ctypes.data, n, -1)
        assert np.allclose(y, np.fft.fft(x), atol=1e-9)
        L.orc_cfft_double(y.ctypes.data, n, 1)
        assert np.allclose(y / n, x, atol=1e-12)


def test_loc_pow_is_corr_loc_pow(oracle):
    """The oracle's local power (-locpow) against corr_loc_pow computed the
    reference's way (src/corr_routines.c:309-366): the double top-hat kernel
    (taps (n/2)/20 at +-6..+-15) correlated with the powers by real FFTs,
    the product scaled by 2/n (real_corr_conv, src/correlations.c), the
    inverse normalised, and the first and last 15 values replaced."""
    rng = np.random.default_rng(41)
    for n in (64, 1024, 4096):
        pw = rng.exponential(1.0, n).astype(np.float32) * (1.0 + np.arange(n) / n)
        kern = np.zeros(n)
        kern[6:16] = (n // 2) // 20
        kern[n - 15:n - 5] = (n // 2) // 20
        corr = np.fft.irfft(np.fft.rfft(pw.astype(np.float64)) * np.conj(np.fft.rfft(kern)), n)
        want = corr * (2.0 / n)
        want[:15] = want[15]
        want[n - 15:] = want[n - 16]
        got = oracle.loc_pow(pw)
        np.testing.assert_allclose(got, want, rtol=2e-7)
        # the mean of 20 neighbours scaled by (2/n) floor(n/40) * 20
        i = n // 2
        direct = (pw[i - 15:i - 5].sum() + pw[i + 6:i + 16].sum()) * ((n // 2) // 20) * 2.0 / n
        assert abs(got[i] - direct) <= 1e-6 * direct
