"""The oracle's f-fdot planes against the reference's own subharm_fderivs_vol
(tests/golden/ref_planes.npz, made by tests/golden/make_ref_planes.py from the
reference's unmodified objects over the FFTW / GSL stand-ins): standard mode,
a jerk search and -locpow, the first and the middle block, every bank the
main loop uses, every 8th z row.  Plane metadata identical; powers within
1e-4 x (power + mean power), the parity suite's plane tolerance (the
reference plane is FP32 with FP32 templates, the oracle's FP64)."""
import importlib.util
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, "golden", "ref_planes.npz"))
ZSTEP = 8


def maker():
    spec = importlib.util.spec_from_file_location(
        "make_ref_accel", os.path.join(HERE, "golden", "make_ref_accel.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def search_kw(opts):
    kw, it = dict(wmax=None, locpow=False), iter(opts)
    for o in it:
        if o in ("-zmax", "-wmax", "-numharm"):
            kw[o[1:]] = int(next(it))
        elif o == "-locpow":
            kw["locpow"] = True
    return kw


def plane_keys(case):
    return sorted({k.rsplit("/", 1)[0] for k in GOLD.files if k.startswith(case + "/")})


def close(dev, ref):
    tol = 1e-4 * (ref + max(float(ref.mean()), 1e-3))
    return bool(np.all(np.abs(dev - ref) <= tol)), float(np.max(np.abs(dev - ref) / (ref + 1.0)))


@pytest.mark.parametrize("case", ["std", "jerk", "std_locpow"])
def test_oracle_planes_match_reference(oracle, case):
    mk = maker()
    N, seed, pulsars, opts = mk.CASES[case]
    fft = mk.spectrum(N, seed, pulsars)
    oobs = oracle.obs_init(oracle.make_params(N, mk.DT, fft.size, **search_kw(opts)))
    banks = {}
    for key in plane_keys(case):
        _, b, nh, hn = key.split("/")
        nh, hn = int(nh), int(hn)
        lo, hi = GOLD[key + "/lohi"]
        if (nh, hn) not in banks:
            banks[(nh, hn)] = oracle.Bank(oobs, nh, hn)
        meta, plane, _, _ = oracle.subharm_fderivs_vol(oobs, fft, nh, hn, float(lo), float(hi),
                                                       banks[(nh, hn)])
        ref = GOLD[key + "/meta"]
        assert [meta[k] for k in ("rlo", "zlo", "wlo", "numrs", "numzs", "numws")] == list(ref), key
        ok, worst = close(plane[:, ::ZSTEP, :], GOLD[key + "/rows"])
        assert ok, (key, worst)
