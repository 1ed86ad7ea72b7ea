"""The device's f-fdot planes (ab_subharm_fderivs_vol) against the reference's
own subharm_fderivs_vol (tests/golden/ref_planes.npz; see
test_cpu_ref_planes.py): standard mode, a jerk search and -locpow, the first
and the middle block, every bank, every 8th z row.  Plane metadata
identical; powers within 1e-4 x (power + mean power)."""
import pytest

from test_cpu_ref_planes import GOLD, ZSTEP, close, maker, plane_keys, search_kw

pytestmark = pytest.mark.gpu
DT = 64e-6


@pytest.mark.parametrize("case", ["std", "jerk", "std_locpow"])
def test_device_planes_match_reference(ctx, ablib, case):
    mk = maker()
    N, seed, pulsars, opts = mk.CASES[case]
    fft = mk.spectrum(N, seed, pulsars)
    obs = ablib.obs_init(ablib.make_params(N, mk.DT, fft.size, **search_kw(opts)))
    ctx.set_spectrum(obs, fft)
    for key in plane_keys(case):
        _, b, nh, hn = key.split("/")
        lo, hi = GOLD[key + "/lohi"]
        meta, plane = ctx.subharm_fderivs_vol(obs, int(nh), int(hn), float(lo), float(hi))
        ref = GOLD[key + "/meta"]
        assert [meta[k] for k in ("rlo", "zlo", "wlo", "numrs", "numzs", "numws")] == list(ref), key
        ok, worst = close(plane[:, ::ZSTEP, :], GOLD[key + "/rows"])
        assert ok, (key, worst)
