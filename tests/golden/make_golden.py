"""Regenerates the golden fixtures in tests/golden/ (run in a container that
has the reference tree; the fixtures travel with the repository).

presto_kats.json
    Known-answer values of PRESTO's own test suite for the Fourier response
    generators (tests/test_presto_python.py:117-146 of the reference),
    transcribed from that file: centre-bin powers of gen_r_response (1.0),
    gen_z_response (z=5, 0.227675) and gen_w_response (z=5, w=40, 0.019462)
    at numbetween=16 with numkern = 2*16*max half width, checked to 6
    decimal places there.
fresnel_ref.npz
    Fresnel integrals S(x), C(x) from the reference's own src/fresnl.c,
    compiled unmodified into oracle/_ref/ by oracle/build_ref.sh, at seeded
    sample points spanning the ranges gen_z_response evaluates.
"""
import ctypes as C
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("PRESTO_REF", "/root/reference")


def kats():
    src = open(os.path.join(REF, "tests", "test_presto_python.py")).read()
    nb = int(re.search(r"^numbetween = (\d+)", src, re.M).group(1))
    z = float(re.search(r"^z = ([\d.]+)", src, re.M).group(1))
    w = float(re.search(r"^w = ([\d.]+)", src, re.M).group(1))
    pz = float(re.search(r"round\(pz\[nn // 2\] - ([\d.]+), (\d+)\)", src).group(1))
    pw = float(re.search(r"round\(pw\[nn // 2\] - ([\d.]+), (\d+)\)", src).group(1))
    places = int(re.search(r"round\(pz\[nn // 2\] - [\d.]+, (\d+)\)", src).group(1))
    pr = float(re.search(r"assert pr\[nn // 2\] == ([\d.]+)", src).group(1))
    return dict(source="tests/test_presto_python.py:117-146", numbetween=nb, z=z, w=w,
                centre_power_r=pr, centre_power_z=pz, centre_power_w=pw, decimals=places)


def fresnel_table():
    sys.path.insert(0, ROOT)
    import subprocess
    subprocess.run(["sh", os.path.join(ROOT, "oracle", "build_ref.sh")], check=True)
    from oracle import pyoracle
    L = pyoracle.ref_fresnel_lib()
    rng = np.random.default_rng(20251203)
    xs = np.concatenate([np.linspace(-3.0, 3.0, 241), rng.uniform(-50, 50, 400),
                         rng.uniform(-800, 800, 200), [0.0, 1.6, 1.8, 2.5625 ** 0.5]])
    S = np.zeros_like(xs)
    Cc = np.zeros_like(xs)
    for i, x in enumerate(xs):
        s, c = C.c_double(), C.c_double()
        L.fresnl(float(x), C.byref(s), C.byref(c))
        S[i], Cc[i] = s.value, c.value
    return xs, S, Cc


if __name__ == "__main__":
    with open(os.path.join(HERE, "presto_kats.json"), "w") as f:
        json.dump(kats(), f, indent=1)
    xs, S, Cc = fresnel_table()
    np.savez_compressed(os.path.join(HERE, "fresnel_ref.npz"), x=xs, S=S, C=Cc,
                        source="reference src/fresnl.c via oracle/build_ref.sh")
    print("wrote", os.listdir(HERE))
