"""Runs the reference's own accelsearch program on seeded synthetic spectra and
keeps its output files as fixtures under tests/golden/ref_accel/<case>/.

The program is src/accelsearch.c with the libpresto files it links, compiled
unmodified into oracle/_ref/accelsearch by oracle/build_ref.sh; FFTW, GSL,
glib and ERFA, which this image lacks, are replaced by stand-ins written for
this repository (oracle/refshim/).  Run here, where the reference tree is;
the fixtures travel with the repository.

Usage: python tests/golden/make_ref_accel.py [case ...] (all cases when none
is named; the manifest keeps the other cases' entries).

Per case: the .fft input is presto_b200.synth's seeded spectrum, or for the
.dat cases its seeded time series (the SHA-256 of the input is recorded so
that a test can confirm it regenerated it; a zap list's text is kept in the
manifest), the
.inf is a telescope "None (Artificial Data Set)" observation, and the
program's three outputs are kept: <root>_ACCEL_<zmax>[_JERK_<wmax>] (text),
.cand (fourierprops records) and .txtcand (one line per candidate insertion
during the search), with its command line in manifest.json.
"""
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "ref_accel")
PROG = os.path.join(ROOT, "oracle", "_ref", "accelsearch")
DT = 64e-6

# name: (N, seed, pulsars, accelsearch options)
CASES = {
    "std": (1 << 17, 11, [dict(r=1500.3, z=12.0, harms=[(0.08, 0.3), (0.05, 1.0), (0.03, 2.0)])],
            ["-zmax", "60", "-wmax", "0", "-numharm", "4"]),
    "inmem": (1 << 17, 12, [dict(r=2222.7, z=-20.0, harms=[(0.06, 0.1)] * 6)],
              ["-zmax", "60", "-numharm", "8"]),
    "jerk": (1 << 16, 13, [dict(r=900.2, z=6.0, w=25.0, harms=[(0.12, 0.0), (0.06, 0.5)])],
             ["-zmax", "20", "-wmax", "40", "-numharm", "2"]),
    "std_locpow": (1 << 17, 14,
                   [dict(r=1700.6, z=-9.0, harms=[(0.08, 0.2), (0.05, 0.9)])],
                   ["-zmax", "60", "-wmax", "0", "-numharm", "4", "-locpow"]),
    # the plain search the benchmarks quote on the CPU-runnable size: N = 2^20,
    # f = 123.4 Hz, z = 40, A = 0.05 (presto_b200.synth.cfg1_spectrum), in memory
    "cfg1": (1 << 20, 1000, [dict(r=123.4 * (1 << 20) * DT, z=40.0, w=0.0, harms=[(0.05, 0.0)])],
             ["-zmax", "200", "-numharm", "8"]),
    # the larger search's parameters (zmax 600, 16 harmonics, standard mode) on
    # N = 2^20: presto_b200.synth.cfg2_spectrum's three 8-harmonic pulsars
    "cfg2s": (1 << 20, 2000, "cfg2", ["-zmax", "600", "-numharm", "16"]),
    # the jerk search's parameters (zmax 200, wmax 300, 8 harmonics) on N = 2^18:
    # presto_b200.synth.cfg3_spectrum's two 4-harmonic sinusoids
    "cfg3s": (1 << 18, 3000, "cfg3", ["-zmax", "200", "-wmax", "300", "-numharm", "8"]),
    # -photon: Poisson counts at 4 per bin, 10 % modulated at r = 3100.4, z = 15;
    # the spectrum is the raw transform, so nph = its DC term
    "photon": (1 << 16, 15, "photon", ["-zmax", "40", "-numharm", "2", "-photon"]),
    "noharmpolish": (1 << 17, 11,
                     [dict(r=1500.3, z=12.0, harms=[(0.08, 0.3), (0.05, 1.0), (0.03, 2.0)])],
                     ["-zmax", "60", "-wmax", "0", "-numharm", "4", "-noharmpolish"]),
    # a .dat time series (realfft + deredden inside accelsearch) with a zap
    # list: a mains line, the injected pulsar's second harmonic (37.3 Hz
    # fundamental, r ~ 625.8), a barycentric birdie, a narrow one widened to
    # a bin, a wide one, one with no room below and one running past Nyquist
    "datzap": (1 << 18, 16, [dict(r=37.3 * (1 << 18) * DT, z=8.0,
                                  harms=[(0.08, 0.2), (0.08, 1.3), (0.06, 2.1), (0.05, 0.7)])],
               ["-zmax", "60", "-numharm", "4", "-zaplist", "datzap.zaplist"]),
    # a 2^7 3^3 5^2 7-sample time series (a typical dedispersed length), its
    # realfft not of a power-of-two length, with two birdies
    "dat7": (604800, 17, [dict(r=88.8 * 604800 * DT, z=-5.0,
                               harms=[(0.07, 0.0), (0.05, 1.1), (0.04, 2.0)])],
             ["-zmax", "40", "-numharm", "2", "-zaplist", "dat7.zaplist"]),
}
# inputs other than a seeded .fft: name -> {"dat": True} (the time series is
# written as <name>.dat) and "zaplist": the text of <name>.zaplist
INPUTS = {
    "datzap": dict(dat=True, zaplist="# birdies for the .dat zapping case (Hz, width Hz)\n"
                                      "50.0 0.1\n74.6 0.2\nB1234.5 0.05\n2000.0 0.01\n"
                                      "3100.0 4.0\n1.0 0.2\n7811.5 3.0\n"),
    "dat7": dict(dat=True, zaplist="60.0 0.1\n266.4 0.3\n"),
}


def inf_text(name, N, dt):
    return (f" Data file name without suffix          =  {name}\n"
            f" Telescope used                         =  None (Artificial Data Set)\n"
            f" Number of bins in the time series      =  {N:<11.0f}\n"
            f" Width of each time series bin (sec)    =  {dt:.15g}\n"
            f" Any breaks in the data? (1 yes, 0 no)  =  0\n"
            f" Data analyzed by                       =  synthetic\n"
            f" Any additional notes:\n"
            f"    seeded synthetic spectrum\n")


def series(N, seed, pulsars):
    """the float32 time series of a .dat case"""
    sys.path.insert(0, ROOT)
    from presto_b200 import synth
    return synth.time_series(N, seed, pulsars).astype(np.float32)


def spectrum(N, seed, pulsars):
    """pulsars: injected signals, "cfg2" / "cfg3" for synth's cfg2/cfg3 draws, or
    "photon" for photon counts (raw transform, PRESTO's packing)"""
    sys.path.insert(0, ROOT)
    from presto_b200 import synth
    if pulsars == "cfg2":
        return synth.cfg2_spectrum(N=N, dt=DT, seed=seed)[0].astype(np.complex64)
    if pulsars == "cfg3":
        return synth.cfg3_spectrum(N=N, dt=DT, seed=seed)[0].astype(np.complex64)
    if pulsars == "photon":
        rng = np.random.default_rng(seed)
        u = np.arange(N) / N
        rate = 4.0 * (1.0 + 0.1 * np.cos(2.0 * np.pi * u * (3100.4 - 7.5 + 7.5 * u)))
        x = rng.poisson(rate).astype(np.float32)
        f = np.fft.rfft(x.astype(np.float64))
        out = f[:N // 2].astype(np.complex64)
        out[0] = complex(f[0].real, f[N // 2].real)
        return out
    return synth.spectrum(synth.time_series(N, seed, pulsars)).astype(np.complex64)


def main():
    if not os.path.exists(PROG):
        subprocess.run(["sh", os.path.join(ROOT, "oracle", "build_ref.sh")], check=True)
    mpath = os.path.join(OUT, "manifest.json")
    manifest = json.load(open(mpath)) if os.path.exists(mpath) else {}
    only = set(sys.argv[1:])
    for name, (N, seed, pulsars, opts) in CASES.items():
        if only and name not in only:
            continue
        extra = INPUTS.get(name, {})
        data = series(N, seed, pulsars) if extra.get("dat") else spectrum(N, seed, pulsars)
        suffix = ".dat" if extra.get("dat") else ".fft"
        with tempfile.TemporaryDirectory() as tmp:
            root = os.path.join(tmp, name)
            data.tofile(root + suffix)
            with open(root + ".inf", "w") as f:
                f.write(inf_text(name, N, DT))
            if "zaplist" in extra:
                with open(root + ".zaplist", "w") as f:
                    f.write(extra["zaplist"])
            r = subprocess.run([PROG] + opts + [name + suffix], cwd=tmp, capture_output=True,
                               text=True, timeout=3600)
            if r.returncode:
                raise RuntimeError(f"{name}: accelsearch exited {r.returncode}\n{r.stdout[-2000:]}")
            dst = os.path.join(OUT, name)
            shutil.rmtree(dst, ignore_errors=True)
            os.makedirs(dst)
            outs = sorted(f for f in os.listdir(tmp) if "_ACCEL_" in f)
            for f in outs:
                shutil.copy(os.path.join(tmp, f), dst)
        manifest[name] = dict(N=N, seed=seed, dt=DT, pulsars=pulsars, options=opts,
                              fft_sha256=hashlib.sha256(data.tobytes()).hexdigest(), files=outs,
                              **extra)
        print(name, outs)
    with open(mpath, "w") as f:
        json.dump(dict(sorted(manifest.items())), f, indent=1)


if __name__ == "__main__":
    main()
