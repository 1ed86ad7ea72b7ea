"""Keeps f-fdot planes of the reference's own subharm_fderivs_vol as fixtures
(tests/golden/ref_planes.npz) for plane-level parity.

oracle/_ref/libref_accel.so (oracle/refdrv.c over the reference's unmodified
objects, FFTW / GSL / glib replaced by the stand-ins of oracle/refshim/)
parses accelsearch's options with the reference's parser and builds the
search with create_accelobs and create_subharminfos.  Per case of
tests/golden/make_ref_accel.py listed below, on its seeded spectrum: the
first and the middle block of the main loop, every bank the loop uses
(harmonic h / n for each stage), every 8th z row (all w and r) to keep the
file small.  Run here, where the reference tree is.
"""
import ctypes as C
import importlib.util
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
CASES = ("std", "jerk", "std_locpow")
ZSTEP = 8


def _maker():
    spec = importlib.util.spec_from_file_location("make_ref_accel",
                                                  os.path.join(HERE, "make_ref_accel.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def main():
    import sys
    sys.path.insert(0, ROOT)
    from oracle import pyoracle
    L = pyoracle.ref_accel_lib()
    if L is None:
        subprocess.run(["sh", os.path.join(ROOT, "oracle", "build_ref.sh")], check=True)
        L = pyoracle.ref_accel_lib()
    mk = _maker()
    arrays = {}
    for name in CASES:
        N, seed, pulsars, opts = mk.CASES[name]
        fft = mk.spectrum(N, seed, pulsars)
        with tempfile.TemporaryDirectory() as tmp:
            root = os.path.join(tmp, name)
            fft.tofile(root + ".fft")
            with open(root + ".inf", "w") as f:
                f.write(mk.inf_text(name, N, mk.DT))
            argv = [b"accelsearch"] + [o.encode() for o in opts] + [(root + ".fft").encode()]
            L.refdrv_open(len(argv), (C.c_char_p * len(argv))(*argv))
            g = (C.c_double * 5)()
            L.refdrv_geometry(g)
            rlo, highestbin, rstep, stages = g[0], g[1], g[2], int(g[3])
            starts = []
            startr = rlo
            while startr + rstep < highestbin:
                starts.append(startr)
                startr += rstep
            for b in sorted({0, len(starts) // 2}):
                lo, hi = starts[b], starts[b] + rstep - 0.5
                banks = [(1, 1)] + [(1 << s, h) for s in range(1, stages) for h in range(1, 1 << s, 2)]
                for nh, hn in banks:
                    meta, p = pyoracle.ref_plane(L, nh, hn, lo, hi)
                    key = f"{name}/{b}/{nh}/{hn}"
                    arrays[key + "/meta"] = np.array([meta[k] for k in ("rlo", "zlo", "wlo", "numrs",
                                                                         "numzs", "numws")])
                    arrays[key + "/lohi"] = np.array([lo, hi])
                    arrays[key + "/rows"] = np.ascontiguousarray(p[:, ::ZSTEP, :])
            L.refdrv_close()
        print(name, "done")
    np.savez_compressed(os.path.join(HERE, "ref_planes.npz"), **arrays)


if __name__ == "__main__":
    main()
