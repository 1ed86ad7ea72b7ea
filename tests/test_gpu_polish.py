"""Device candidate polishing (ab_optimize_cands) against the reference's
optimizer battery and against the polishing oracle.

* The battery of the reference's tests/test_maximize_rz.py (restated in
  test_cpu_polish.py), through the C ABI, with the reference's tolerances.
* Agreement with the oracle: both run the same two Nelder-Mead stages to a
  1e-7 size tolerance; the amplitudes differ in summation order (float in the
  reference and the oracle, FP64 per warp on the device), so the optimum
  agrees to ~1e-4 bins: |dr| <= 2e-3 bins, |dz| <= 1e-2, the summed power
  of the harmonics within 1e-3 relative, each harmonic's power within
  1e-3 relative plus twice its slope times the difference of the optima, local
  powers within 1e-3 relative or 1e-6 of the peak power.
* Candidates of a real search (cfg1 recipe at N = 2^19): the same bounds.
"""
import numpy as np
import pytest

from presto_b200 import synth
from test_cpu_polish import (HARM_OFFSETS, HARM_Z_VALUES, N, NOISE_CASES, R_HARM, R_RZ,
                             RZ_OFFSETS, THEO_POW, TOL, Z_VALUES, _check, harmonic_signal)

pytestmark = pytest.mark.gpu
DT = 64e-6


def _obs(ablib, numbins):
    return ablib.obs_init(ablib.make_params(N, DT, numbins, zmax=100, wmax=0, numharm=4))


def _agree(dev, orc, tag):
    for k, (d, o) in enumerate(zip(dev, orc)):
        info = (tag, k, d["hirs"], o["hirs"], d["hizs"], o["hizs"], d["pows"], o["pows"])
        assert np.max(np.abs(d["hirs"] - o["hirs"])) <= 2e-3, info
        assert np.max(np.abs(d["hizs"] - o["hizs"])) <= 1e-2, info
        # the summed power is flat at the optimum (the quantity the reference's
        # battery checks); a single harmonic on the slope of its peak moves by
        # its slope times the small difference of the optima
        assert abs(np.sum(d["pows"]) - np.sum(o["pows"])) <= 1e-3 * np.sum(o["pows"]), info
        slope = np.abs(o["derivs"][:, 2]) * np.abs(d["hirs"] - o["hirs"])
        assert np.all(np.abs(d["pows"] - o["pows"]) <= 1e-3 * np.abs(o["pows"]) + 2 * slope), info
        # local powers: relative, or against the peak where they are tiny
        # (the sidelobes of a noiseless tone, 1e-10 of the peak)
        assert np.allclose(d["derivs"][:, 6], o["derivs"][:, 6], rtol=1e-3,
                           atol=1e-6 * np.max(o["pows"])), info


@pytest.mark.parametrize("noise_amp,seed", NOISE_CASES)
def test_device_polish_battery_single(ctx, ablib, oracle, noise_amp, seed):
    fails = []
    for z in Z_VALUES:
        ft = harmonic_signal(R_RZ, z, 1, noise_amp, seed)
        obs = _obs(ablib, ft.size)
        cands = [(0.0, 0.0, 1, R_RZ + dr, z + dz, 0.0) for dr, dz in RZ_OFFSETS]
        dev = ctx.optimize_cands(obs, ft, cands)
        orc = oracle.optimize_cands(ft, 0, [(1, c[3], c[4]) for c in cands])
        _agree(dev, orc, ("single", z))
        for c, d in zip(cands, dev):
            if not _check(TOL[noise_amp], d["hirs"][0] - R_RZ, d["hizs"][0] - z,
                          d["pows"][0] / THEO_POW):
                fails.append((z, c[3], c[4], d["hirs"][0], d["hizs"][0], d["pows"][0] / THEO_POW))
    assert not fails, fails


@pytest.mark.parametrize("numharm", [2, 3, 4])
@pytest.mark.parametrize("noise_amp,seed", NOISE_CASES)
def test_device_polish_battery_harmonics(ctx, ablib, oracle, numharm, noise_amp, seed):
    fails = []
    for z in HARM_Z_VALUES:
        ft = harmonic_signal(R_HARM, z, numharm, noise_amp, seed)
        obs = _obs(ablib, ft.size)
        cands = [(0.0, 0.0, numharm, R_HARM + dr, z + dz, 0.0) for dr, dz in HARM_OFFSETS]
        dev = ctx.optimize_cands(obs, ft, cands)
        orc = oracle.optimize_cands(ft, 0, [(numharm, c[3], c[4]) for c in cands])
        _agree(dev, orc, ("harm", numharm, z))
        for c, d in zip(cands, dev):
            maxpow = d["derivs"][:, 0].sum()
            if not _check(TOL[noise_amp], d["hirs"][0] - R_HARM, d["hizs"][0] - z,
                          maxpow / (numharm * THEO_POW)):
                fails.append((z, c[3], c[4], d["hirs"][0], d["hizs"][0]))
    assert not fails, fails


def test_device_polish_search_candidates(ctx, ablib, oracle):
    """Polish the candidates of a cfg1-recipe search (N = 2^19, zmax 200, 8
    harmonics) on the device and in the oracle."""
    n = 1 << 19
    fft = synth.cfg1_spectrum(N=n, amp=0.05)
    obs = ablib.obs_init(ablib.make_params(n, DT, fft.size, zmax=200, numharm=8))
    cands = ctx.search(obs, fft)
    assert len(cands) > 0
    cands = sorted(cands, key=lambda c: -c[1])[:24]
    dev = ctx.optimize_cands(obs, fft, cands)
    orc = oracle.optimize_cands(fft, obs.lobin, [(c[2], c[3], c[4]) for c in cands], nthreads=8)
    _agree(dev, orc, "search")


def test_device_noharmpolish_accel(ctx, ablib, oracle):
    """-noharmpolish: max_rz_arr for every harmonic on its own at (r n, z n)
    (src/accel_utils.c:598-611), device against the oracle's max_rz_arr."""
    fails = []
    for z in HARM_Z_VALUES:
        ft = harmonic_signal(R_HARM, z, 3, 1.0, 4321)
        obs = ablib.obs_init(ablib.make_params(N, DT, ft.size, zmax=100, wmax=0, numharm=4,
                                               noharmpolish=True))
        assert obs.noharmpolish == 1
        dr, dz = HARM_OFFSETS[1]
        dev = ctx.optimize_cands(obs, ft, [(0.0, 0.0, 3, R_HARM + dr, z + dz, 0.0)])[0]
        for ii in range(3):
            n = ii + 1
            p, ro, zo, rd = oracle.max_rz_arr(ft, (R_HARM + dr) * n, (z + dz) * n)
            ok = (abs(dev["hirs"][ii] - ro) <= 2e-3 and abs(dev["hizs"][ii] - zo) <= 1e-2 and
                  abs(dev["pows"][ii] - p) <= 1e-3 * p and
                  # local power: relative, or against the peak (the 20 points sit at
                  # integer offsets from each side's optimum, which differ by ~1e-4
                  # bins, so a strong tone's leakage into them differs), as _agree
                  abs(dev["derivs"][ii][6] - rd.locpow) <= 1e-3 * rd.locpow + 1e-6 * p)
            if not ok:
                fails.append(f"z={z} n={n} r {dev['hirs'][ii]!r} {ro!r} z {dev['hizs'][ii]!r} {zo!r} "
                             f"pow {dev['pows'][ii]!r} {p!r} locpow {dev['derivs'][ii][6]!r} "
                             f"{rd.locpow!r}")
    assert not fails, fails
