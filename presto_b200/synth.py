"""Seeded synthetic .fft spectra for the search workloads.

A float32 N(0,1) time series plus injected pulsars is real-FFT'd and packed
like PRESTO's realfft (src/fastffts.c:163-258): N/2 complex bins with bin 0
holding (DC, Nyquist).  Amplitudes are scaled so that the mean noise power
is 1.  Injections use the mid-observation parametrisation of PRESTO's
tests/test_max_rzw_harmonics.py:27-35: for u = t/T, harmonic k has phase
2 pi k (u (u (u w/6 + z0/2) + r0)) with r0 = r - z/2 + w/12, z0 = z - w/2,
so r, z and w are averages over the observation.
"""
import numpy as np


def time_series(N, seed, pulsars=(), dtype=np.float32):
    """pulsars: iterable of dicts with r, z, w (fundamental, in bins) and
    harms: list of (amplitude, phase) per harmonic."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(N).astype(np.float64)
    if pulsars:
        u = np.arange(N, dtype=np.float64) / N
        for p in pulsars:
            r, z, w = p["r"], p.get("z", 0.0), p.get("w", 0.0)
            r0, z0 = r - z / 2.0 + w / 12.0, z - w / 2.0
            base = u * (u * (u * w / 6.0 + z0 / 2.0) + r0)
            for k, (amp, phs) in enumerate(p["harms"], start=1):
                x += amp * np.cos(2.0 * np.pi * k * base + phs)
    return x.astype(dtype)


def spectrum(x):
    """PRESTO-packed, unit-mean-noise-power spectrum (complex64, N/2 bins)."""
    N = x.size
    X = np.fft.rfft(x.astype(np.float64))
    out = np.empty(N // 2, np.complex64)
    out[:] = X[:N // 2] / np.sqrt(N)
    out[0] = complex(X[0].real / np.sqrt(N), X[N // 2].real / np.sqrt(N))
    return out


def cfg1_spectrum(N=1 << 20, dt=64e-6, seed=1000, f=123.4, z=40.0, amp=0.05):
    """Plain search, one sinusoid with constant acceleration."""
    T = N * dt
    p = dict(r=f * T, z=z, w=0.0, harms=[(amp, 0.0)])
    return spectrum(time_series(N, seed, [p]))


def cfg2_spectrum(N=1 << 23, dt=64e-6, seed=2000):
    """Larger acceleration search: 3 pulsars, 8 harmonics at 0.02 each,
    f log-uniform in 2-700 Hz, z uniform in [-500, 500]."""
    rng = np.random.default_rng(seed + 1)
    T = N * dt
    ps = []
    for _ in range(3):
        f = float(np.exp(rng.uniform(np.log(2.0), np.log(700.0))))
        z = float(rng.uniform(-500, 500))
        harms = [(0.02, float(rng.uniform(0, 2 * np.pi))) for _ in range(8)]
        ps.append(dict(r=f * T, z=z, w=0.0, harms=harms))
    return spectrum(time_series(N, seed, ps)), ps


def cfg3_spectrum(N=1 << 22, dt=64e-6, seed=3000):
    """Jerk search: 2 sinusoids with 4 harmonics, z in [-150,150], w in [-250,250]."""
    rng = np.random.default_rng(seed + 1)
    T = N * dt
    ps = []
    for _ in range(2):
        f = float(np.exp(rng.uniform(np.log(5.0), np.log(500.0))))
        ps.append(dict(r=f * T, z=float(rng.uniform(-150, 150)), w=float(rng.uniform(-250, 250)),
                       harms=[(0.03, float(rng.uniform(0, 2 * np.pi))) for _ in range(4)]))
    return spectrum(time_series(N, seed, ps)), ps
