"""The polishing oracle (oracle/polish_oracle.c) against the reference's own
optimizer battery, tests/test_maximize_rz.py of the reference: sinusoids
injected at known Fourier (r, z) in N = 2^14 samples, the optimizers started
from perturbed points, the recovered peak location and power checked against
the reference's tolerances (noiseless: |dr| < 0.01, |dz| < 0.03, power within
1 %; unit-variance noise: |dr| < 0.05, |dz| < 0.20, power 0.90-1.12 of
theory).  The battery's cases, offsets and tolerances are the reference's;
the spectra are numpy real FFTs packed as PRESTO's realfft packs them (bin 0
= DC, Nyquist)."""
import numpy as np
import pytest

N = 2 ** 14
R_RZ = N / 4.0
R_HARM = N / 16.0
THEO_POW = N ** 2.0 / 4.0
RZ_OFFSETS = [(0.0, 0.0), (0.12, -0.8), (-0.2, 1.3), (0.3, 2.0), (-0.35, -2.5)]
HARM_OFFSETS = [(0.0, 0.0), (0.15, 1.0), (-0.25, -1.5)]
Z_VALUES = [0.0, 1.0, 2.5, 5.0, -5.0, 10.0, -10.0, 30.0, -30.0, 55.0]
HARM_Z_VALUES = [0.0, 5.0, -8.0, 20.0]
NOISE_CASES = [(0.0, 0), (1.0, 12345)]
TOL = {0.0: dict(dr=0.01, dz=0.03, plo=0.99, phi=1.01),
       1.0: dict(dr=0.05, dz=0.20, plo=0.90, phi=1.12)}


def presto_rfft(sig):
    x = np.fft.rfft(sig)
    out = x[:sig.size // 2].astype(np.complex64)
    out[0] = complex(x[0].real, x[sig.size // 2].real)
    return out


def harmonic_signal(r, z, numharm, noise_amp=0.0, seed=0):
    us = np.arange(N, dtype=np.float64) / N
    sig = np.zeros(N)
    for h in range(1, numharm + 1):
        rh, zh = r * h, z * h
        sig += np.cos(2.0 * np.pi * (us * (us * (zh / 2.0) + (rh - 0.5 * zh))))
    if noise_amp:
        sig = sig + noise_amp * np.random.default_rng(seed).standard_normal(N)
    return presto_rfft(sig)


def _check(tol, dr, dz, pf):
    return abs(dr) <= tol["dr"] and abs(dz) <= tol["dz"] and tol["plo"] <= pf <= tol["phi"]


@pytest.mark.parametrize("noise_amp,seed", NOISE_CASES)
def test_max_rz_arr_recovers_injected_peaks(oracle, noise_amp, seed):
    fails = []
    for z in Z_VALUES:
        ft = harmonic_signal(R_RZ, z, 1, noise_amp, seed)
        for dr, dz in RZ_OFFSETS:
            p, ro, zo, _ = oracle.max_rz_arr(ft, R_RZ + dr, z + dz)
            if not _check(TOL[noise_amp], ro - R_RZ, zo - z, p / THEO_POW):
                fails.append((z, dr, dz, ro - R_RZ, zo - z, p / THEO_POW))
    assert not fails, fails


@pytest.mark.parametrize("numharm", [2, 3, 4])
@pytest.mark.parametrize("noise_amp,seed", NOISE_CASES)
def test_max_rz_arr_harmonics_recovers_injected_peaks(oracle, numharm, noise_amp, seed):
    fails = []
    for z in HARM_Z_VALUES:
        ft = harmonic_signal(R_HARM, z, numharm, noise_amp, seed)
        for dr, dz in HARM_OFFSETS:
            ro, zo, rds, _ = oracle.max_rz_arr_harmonics(ft, R_HARM + dr, z + dz, numharm)
            maxpow = sum(rd.pow for rd in rds)
            if not _check(TOL[noise_amp], ro - R_HARM, zo - z, maxpow / (numharm * THEO_POW)):
                fails.append((z, dr, dz, ro - R_HARM, zo - z, maxpow / (numharm * THEO_POW)))
    assert not fails, fails


def test_rz_interp_exact_at_bins_and_symmetric(oracle):
    """At integer r and z = 0 the interpolation returns the bin itself
    (src/rzinterp.c:181-192); for a tone half-way between bins it is
    symmetric about the tone, and the peak power approaches N^2/4 as the
    kernel widens (truncated sinc tails: 0.97 at 16 bins, within 1 % at the
    HIGHACC width 48, within 0.3 % at 200)."""
    ft = harmonic_signal(R_RZ + 0.5, 0.0, 1)
    k = int(R_RZ)
    assert oracle.rz_interp(ft, float(k), 0.0, 32) == complex(ft[k])
    fr = []
    for hw in (16, 48, 200):
        lo = abs(oracle.rz_interp(ft, R_RZ + 0.25, 0.0, hw))
        hi = abs(oracle.rz_interp(ft, R_RZ + 0.75, 0.0, hw))
        peak = abs(oracle.rz_interp(ft, R_RZ + 0.5, 0.0, hw))
        assert abs(lo - hi) <= 1e-4 * peak and peak > lo
        fr.append(peak ** 2 / THEO_POW)
    assert fr[0] < fr[1] < fr[2] <= 1.0
    assert fr[1] > 0.99 and fr[2] > 0.997


def test_calc_props_of_a_polished_tone(oracle):
    """calc_props on the derivatives at a recovered peak: normalised power =
    raw / local power, error estimates positive and finite."""
    ft = harmonic_signal(R_RZ, 10.0, 1, 1.0, 7)
    p, ro, zo, rd = oracle.max_rz_arr(ft, R_RZ + 0.1, 10.5)
    props = oracle.FourierProps()
    L = oracle._polish_lib()
    assert L.orc_calc_props(rd, ro, zo, 0.0, props) == 0
    assert abs(props.pow - rd.pow / rd.locpow) <= 1e-6 * props.pow
    assert props.rawpow == pytest.approx(rd.pow, rel=1e-6)
    for f in ("rerr", "zerr", "powerr", "pur", "sig"):
        assert np.isfinite(getattr(props, f)) and getattr(props, f) > 0
