"""The oracle and the product's host functions against the reference's own
code, compiled here from its unmodified sources by oracle/build_ref.sh
(src/characteristics.c, rzinterp.c, rzwinterp.c, responses.c, fresnl.c,
vectors.c with the reference's own realfft and fftwcall, over the FFTW / GSL
stand-ins of oracle/refshim/: FFTW's plans run an FP64 transform).  Skipped
when the reference tree is absent.

* gen_r_response / gen_z_response / gen_w_response (src/responses.c:159-418)
  against the oracle's restatements: within 2e-6 of the response's peak (the
  tolerance the device templates are held to against the oracle).
* z_resp_halfwidth / w_resp_halfwidth (src/responses.c:27-84): the product's
  ab_w_resp_halfwidth and the oracle's, identical integers.
* rz_interp / rzw_interp (src/rzinterp.c:144-236, src/rzwinterp.c:145-229),
  get_localpower3d and get_derivs3d (src/characteristics.c:79-192): the
  oracle's polishing primitives within 1e-5 relative (powers, local powers),
  1e-4 (first derivatives) and float rounding amplified by the second
  difference's 1/(2h)^2 (second derivatives).
* calc_props / calc_rzwerrs (src/characteristics.c:195-264, 353-392): the
  product's ab_calc_props / ab_calc_rzwerrs bit for bit.
"""
import ctypes as C  # noqa: N812

import numpy as np
import pytest

LOWACC, HIGHACC = 0, 1


@pytest.fixture(scope="module")
def ref(oracle):
    L = oracle.ref_polish_lib()
    if L is None:
        pytest.skip("reference sources not built here (oracle/build_ref.sh)")
    return L


@pytest.mark.parametrize("kind,nb,z,w,roff", [
    ("r", 2, 0.0, 0.0, 0.0), ("r", 16, 0.0, 0.0, 0.37), ("r", 1, 0.0, 0.0, 0.9),
    ("z", 2, 0.0, 0.0, 0.0), ("z", 2, 3.0, 0.0, 0.0), ("z", 16, 5.0, 0.0, 0.0),
    ("z", 2, -47.5, 0.0, 0.25), ("z", 2, 200.0, 0.0, 0.0), ("z", 1, -600.0, 0.0, 0.6),
    ("z", 8, 1e-5, 0.0, 0.5),
    ("w", 2, 0.0, 40.0, 0.0), ("w", 16, 5.0, 40.0, 0.0), ("w", 2, -60.0, 200.0, 0.0),
    ("w", 2, 100.0, -300.0, 0.0), ("w", 1, 12.3, 86.0, 0.41), ("w", 2, 0.0, 1e-5, 0.0),
])
def test_responses_match_reference(ref, oracle, kind, nb, z, w, roff):
    if kind == "r":
        numkern = 2 * nb * 32
    elif kind == "z":
        numkern = 2 * nb * ref.z_resp_halfwidth(z, LOWACC)
    else:
        numkern = 2 * nb * ref.w_resp_halfwidth(z, w, LOWACC)
    want = oracle.ref_response(ref, kind, nb, numkern, z=z, w=w, roffset=roff)
    got = oracle.response(kind, nb, numkern, z=z, w=w, roffset=roff)
    peak = np.max(np.abs(want))
    zero = numkern // 2 + roff * nb
    if roff > 0.0 and zero == int(zero) and (kind == "r" or abs(z) < 1e-4):
        # the sinc's argument is 0 on the grid: the reference's recursion
        # (src/responses.c:199-211) divides two rounding residues there, the
        # restatement takes the limit, 1
        k = int(zero)
        assert got[k] == 1.0 and abs(want[k]) < 0.5
        got[k] = want[k]
    assert np.max(np.abs(got - want)) <= 2e-6 * peak, (kind, z, w)


def test_halfwidths_match_reference(ref, ablib, oracle):
    L = oracle.lib(64)
    rng = np.random.default_rng(1)
    zs = np.concatenate([[0.0, 1e-5, 2.0, -2.0, 600.0, -1200.0], rng.uniform(-1200, 1200, 300)])
    ws = np.concatenate([[0.0, 1e-5, 20.0, -300.0, 1200.0, 0.0], rng.uniform(-1200, 1200, 300)])
    for z, w in zip(zs.tolist(), ws.tolist()):
        want = ref.w_resp_halfwidth(z, w, LOWACC)
        assert ablib.lib().ab_w_resp_halfwidth(z, w) == want, (z, w)
        assert L.orc_w_resp_halfwidth(z, w) == want, (z, w)
        if w == 0.0:
            assert ref.z_resp_halfwidth(z, LOWACC) == want


def _spectrum(seed, n=1 << 13):
    rng = np.random.default_rng(seed)
    x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    k = np.arange(n)
    x[1000:1100] += (30.0 * np.exp(1j * 0.02 * (k[1000:1100] - 1000) ** 2)).astype(np.complex64)
    return x


def test_interpolators_match_reference(ref, oracle):
    data = _spectrum(2)
    rng = np.random.default_rng(3)
    out = np.zeros(1, np.complex64)
    for _ in range(120):
        r = float(rng.uniform(40, data.size - 40))
        z = float(rng.uniform(-60, 60))
        w = float(rng.choice([0.0, rng.uniform(-250, 250)]))
        acc = int(rng.integers(0, 2))
        if w == 0.0:
            hw = ref.z_resp_halfwidth(z, acc)
            ref.rz_interp(data.ctypes.data, data.size, r, z, hw, out.ctypes.data)
        else:
            hw = ref.w_resp_halfwidth(z, w, acc)
            ref.rzw_interp(data.ctypes.data, data.size, r, z, w, hw, out.ctypes.data)
        want = complex(out[0])
        got = oracle.rz_interp(data, r, z, hw, w=w)
        err = abs(got - want) / (abs(want) + 1.0)
        assert err <= 1e-5, (r, z, w, hw, got, want)


def test_localpower_and_derivs_match_reference(ref, oracle):
    data = _spectrum(4)
    P = oracle._polish_lib()
    rng = np.random.default_rng(5)
    for _ in range(40):
        r = float(rng.uniform(60, data.size - 60))
        z = float(rng.uniform(-40, 40))
        w = float(rng.choice([0.0, rng.uniform(-150, 150)]))
        lp_ref = ref.get_localpower3d(data.ctypes.data, data.size, r, z, w)
        lp = P.orc_get_localpower3d(data.ctypes.data, data.size, r, z, w)
        assert abs(lp - lp_ref) <= 1e-5 * lp_ref, (r, z, w)
        want, got = oracle.RDerivs(), oracle.RDerivs()
        ref.get_derivs3d(data.ctypes.data, data.size, r, z, w, lp_ref, C.byref(want))
        P.orc_get_derivs3d(data.ctypes.data, data.size, r, z, w, lp_ref, C.byref(got))
        scale = want.pow + lp_ref
        assert abs(got.pow - want.pow) <= 1e-5 * scale
        assert abs(got.locpow - want.locpow) == 0.0
        assert abs(np.angle(np.exp(1j * (got.phs - want.phs)))) <= 1e-4 * (1.0 + lp_ref / want.pow)
        assert abs(got.dpow - want.dpow) <= 1e-4 * scale
        # second difference over (2h)^2 = 3.6e-5 (src/characteristics.c:162,189):
        # float rounding (~2e-7) of the four interpolated powers it adds, amplified
        assert abs(got.d2pow - want.d2pow) <= 4 * 2e-7 * scale / 3.6e-5


def test_calc_props_and_rzwerrs_match_reference_bit_for_bit(ref, ablib, oracle):
    rng = np.random.default_rng(6)
    for _ in range(500):
        loc = float(rng.uniform(0.2, 5.0))
        d = [float(rng.uniform(1e-3, 500)) * loc, float(rng.uniform(-np.pi, np.pi)),
             float(rng.normal(0, 20)), float(rng.normal(0, 2)), float(-abs(rng.normal(0, 900))),
             float(rng.normal(0, 2)), loc]
        r, z, w = float(rng.uniform(10, 1e7)), float(rng.normal(0, 150)), float(rng.normal(0, 300))
        want = oracle.FourierProps()
        ref.calc_props(oracle.RDerivs(*d), r, z, w, C.byref(want))
        got = ablib.calc_props(d, r, z, w)
        assert bytes(got) == bytes(want), d
        T = float(rng.uniform(10, 2e4))
        ew = oracle.RzwErrs()
        ref.calc_rzwerrs(C.addressof(want), T, C.addressof(ew))
        eg = ablib.calc_rzwerrs(got, T)
        assert bytes(eg) == bytes(ew), (d, T)
