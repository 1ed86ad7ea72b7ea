"""Device time-series input path against its oracle: realfft at lengths that
take the single-transform, four-pass and four-step routes (FP32 on the device
vs the oracle's FP64 FFT: within 2e-6 of the largest bin), deredden
bit-exact on the same input, the whole chain within 1e-4 of the largest bin,
and a search of the device's spectrum giving the same candidates as a search
of the oracle's."""
import numpy as np
import pytest

from presto_b200 import synth

pytestmark = pytest.mark.gpu
DT = 64e-6


@pytest.mark.parametrize("n", [1 << 12, 1 << 14, 1 << 17, 1 << 21, 1 << 23])
def test_device_realfft(ctx, oracle, n):
    x = np.random.default_rng(n + 1).standard_normal(n).astype(np.float32)
    dev = ctx.realfft(x)
    orc = oracle.realfft(x)
    scale = np.max(np.abs(orc))
    assert np.max(np.abs(dev - orc)) <= 2e-6 * scale


@pytest.mark.parametrize("n", [1026, 67228, 604800, 3888000])
def test_device_realfft_any_even_length(ctx, oracle, n):
    """Lengths that are not powers of two (n/2 = 3^3 19, 2 7^5, 2^6 3^3 5^2 7,
    2^6 3^5 5^3): Bluestein's transform over power-of-two FFTs, against the
    oracle's FP64 mixed-radix FFT."""
    x = np.random.default_rng(n + 3).standard_normal(n).astype(np.float32)
    dev = ctx.realfft(x)
    orc = oracle.realfft(x)
    scale = np.max(np.abs(orc))
    assert np.max(np.abs(dev - orc)) <= 3e-6 * scale, np.max(np.abs(dev - orc)) / scale


def test_device_realfft_prime_half_length(ctx):
    """n/2 = 65537 (prime), against numpy's FP64 transform in the reference's
    packing (bin 0 = DC, Nyquist)."""
    n = 2 * 65537
    x = np.random.default_rng(5).standard_normal(n).astype(np.float32)
    X = np.fft.rfft(x.astype(np.float64))
    want = X[:n // 2].copy()
    want[0] = complex(X[0].real, X[n // 2].real)
    dev = ctx.realfft(x)
    assert np.max(np.abs(dev - want)) <= 3e-6 * np.max(np.abs(want))


def test_series_search_at_a_dedispersed_length(ctx, ablib, oracle):
    """A 2^7 3^3 5^2 7-sample series (604800 samples, a typical dedispersed
    length): the device's series-to-spectrum path and search give the
    candidates of the oracle's path."""
    n = 604800
    series = np.asarray(synth.time_series(n, 77, [dict(r=2100.3, z=6.0, harms=[(0.06, 0.1)] * 2)]),
                        np.float32)
    dev = ctx.series_to_fft(series, DT)
    orc = oracle.deredden(oracle.realfft(series), 6, 200, 0.5 / DT, n * DT)
    assert np.max(np.abs(dev - orc)) <= 1e-4 * np.max(np.abs(orc))
    kw = dict(zmax=20, numharm=2)
    obs = ablib.obs_init(ablib.make_params(n, DT, dev.size, **kw))
    a = ctx.search(obs, dev)
    b = ctx.search(obs, orc)
    assert len(a) == len(b) and len(a) > 0
    for x, y in zip(a, b):
        assert x[2] == y[2] and abs(x[3] - y[3]) < 1e-3 and abs(x[4] - y[4]) < 1e-3


@pytest.mark.parametrize("numbins", [1 << 11, 1 << 16, 1 << 22])
def test_device_deredden_bitexact(ctx, oracle, numbins):
    rng = np.random.default_rng(numbins)
    k = np.arange(1, numbins + 1)
    spec = ((rng.standard_normal(numbins) + 1j * rng.standard_normal(numbins)) *
            (1.0 + 3e3 / k)).astype(np.complex64)
    T = 2 * numbins * DT
    dev = ctx.deredden(spec, 6, 200, 0.5 / DT, T)
    orc = oracle.deredden(spec, 6, 200, 0.5 / DT, T)
    assert np.array_equal(dev.view(np.uint32), orc.view(np.uint32))


def test_series_to_fft_and_search(ctx, ablib, oracle):
    n = 1 << 20
    series = synth.time_series(n, 1000, [dict(r=123.4 * n * DT, z=40.0, harms=[(0.05, 0.0)])])
    series = np.asarray(series, np.float32)
    dev = ctx.series_to_fft(series, DT)
    orc = oracle.deredden(oracle.realfft(series), 6, 200, 0.5 / DT, n * DT)
    assert np.max(np.abs(dev - orc)) <= 1e-4 * np.max(np.abs(orc))
    obs = ablib.obs_init(ablib.make_params(n, DT, dev.size, zmax=200, numharm=8))
    a = ctx.search(obs, dev)
    b = ctx.search(obs, orc)
    assert len(a) == len(b) and len(a) > 0
    for x, y in zip(a, b):
        assert x[2] == y[2] and abs(x[3] - y[3]) < 1e-3 and abs(x[4] - y[4]) < 1e-3
        assert abs(x[0] - y[0]) <= 1e-3 * y[0]


def test_zapbirds_on_device_matches_host(ctx, ablib):
    """-zaplist zapping of a device-resident spectrum (only the windows it
    reads and the bins it writes cross the bus) equals the host routine bit
    for bit, itself pinned against the reference's zapbirds on the CPU."""
    import torch

    n = 1 << 20
    rng = np.random.default_rng(7)
    spec = (rng.standard_normal(n // 2) + 1j * rng.standard_normal(n // 2)).astype(np.complex64)
    lo = np.array([20.0, 3000.2, 3150.0, 70000.0, 262000.0, 524000.5])
    hi = np.array([25.0, 3010.9, 3151.0, 70400.0, 262001.0, 524290.0])
    want = ablib.zapbirds_host(spec, n, lo, hi)
    dev = torch.from_numpy(spec.view(np.float32).copy()).cuda()
    ctx.zapbirds(None, n, lo, hi, device_ptr=dev.data_ptr(), numbins=spec.size)
    got = dev.cpu().numpy().view(np.complex64)
    assert ctx.last_numzapped == 6
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert not np.array_equal(got, spec)


def test_device_pointers_off_their_boundary(ctx, ablib):
    """A device series that starts 4 bytes off an 8-byte boundary (a trial of
    odd length inside a DM-trial array) is read through the aligned input
    buffer and gives the aligned result bit for bit; a device spectrum off its
    8-byte boundary is refused before anything is launched."""
    import ctypes as C

    import torch

    n = 1 << 16
    x = synth.time_series(n, 17, [dict(r=900.3, z=0.0, harms=[(0.2, 0.0)])]).astype(np.float32)
    want = ctx.series_to_fft(x, DT)
    buf = torch.zeros(n + 1, dtype=torch.float32, device="cuda")
    buf[1:] = torch.from_numpy(x).cuda()
    out = torch.empty(n, dtype=torch.float32, device="cuda")     # n/2 complex bins
    rc = ctx.L.ab_series_to_fft(ctx.ptr, C.c_void_p(buf.data_ptr() + 4), n, DT, 1,
                                C.c_void_p(out.data_ptr()), 1)
    assert rc == 0
    got = out.cpu().numpy().view(np.complex64)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    rc = ctx.L.ab_series_to_fft(ctx.ptr, C.c_void_p(buf.data_ptr()), n, DT, 1,
                                C.c_void_p(out.data_ptr() + 4), 1)
    assert rc == -1                                               # AB_ERR_ARG
    obs = ablib.obs_init(ablib.make_params(n, DT, n // 2, zmax=10, numharm=2))
    with pytest.raises(ablib.AccelError):
        ctx.search(obs, None, device_ptr=out.data_ptr() + 4)
    assert len(ctx.search(obs, None, device_ptr=out.data_ptr())) == len(ctx.search(obs, want))
