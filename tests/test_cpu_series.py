"""The time-series input path's oracle (oracle/series_oracle.c): realfft
against numpy's real FFT (bin 0 packed as (DC, Nyquist) as PRESTO packs it),
deredden's effect on white and red noise, and the host plan of its blocks."""
import ctypes as C

import numpy as np
import pytest


@pytest.mark.parametrize("n", [1 << 12, 1 << 17])
def test_oracle_realfft_matches_numpy(oracle, n):
    x = np.random.default_rng(n).standard_normal(n).astype(np.float32)
    f = oracle.realfft(x)
    ref = np.fft.rfft(x.astype(np.float64))
    assert f.size == n // 2
    assert f[0].real == pytest.approx(ref[0].real, rel=1e-6, abs=1e-3)
    assert f[0].imag == pytest.approx(ref[n // 2].real, rel=1e-6, abs=1e-3)
    assert np.max(np.abs(f[1:] - ref[1:n // 2])) <= 1e-6 * np.max(np.abs(ref))


def test_oracle_deredden_flattens_red_noise(oracle):
    n = 1 << 18
    dt = 64e-6
    rng = np.random.default_rng(3)
    k = np.arange(1, n // 2 + 1)
    spec = (rng.standard_normal(n // 2) + 1j * rng.standard_normal(n // 2)) * (1.0 + 2e4 / k)
    spec = spec.astype(np.complex64)
    d = oracle.deredden(spec, 6, 200, 0.5 / dt, n * dt)
    assert d[0] == 1.0 + 0.0j
    p = np.abs(d[1:]) ** 2
    lo, hi = p[: p.size // 8].mean(), p[-p.size // 8:].mean()
    assert 0.9 < lo < 1.1 and 0.9 < hi < 1.1
    raw = np.abs(spec[1:]) ** 2
    assert raw[: raw.size // 8].mean() > 10 * raw[-raw.size // 8:].mean()


def test_dered_plan_partitions_the_spectrum(ablib):
    """Blocks follow each other from bin 1 to the end; lengths start at
    startwidth and grow as startwidth ln(bin), capped at endwidth."""
    L = ablib.lib()
    f = L.ab_dered_plan
    f.argtypes = [C.c_longlong, C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p,
                  C.c_longlong, C.POINTER(C.c_longlong)]
    numbins = 1 << 20
    nb = C.c_longlong()
    assert f(numbins, 6, 200, 1e300, 1.0, None, 0, C.byref(nb)) == 0
    blocks = np.zeros((nb.value, 2), np.int32)
    assert f(numbins, 6, 200, 1e300, 1.0, blocks.ctypes.data, nb.value, C.byref(nb)) == 0
    assert blocks[0, 0] == 1 and blocks[0, 1] == 6
    assert np.all(blocks[1:, 0] == blocks[:-1, 0] + blocks[:-1, 1])
    assert blocks[-1, 0] + blocks[-1, 1] == numbins
    binnum = 1 + np.cumsum(blocks[:, 1])
    want = np.minimum((6 * np.log(binnum[:-1].astype(np.float64))).astype(int), 200)
    assert np.array_equal(blocks[1:-1, 1], want[:-1])
    assert f(5, 6, 200, 1e300, 1.0, None, 0, C.byref(nb)) == -1
