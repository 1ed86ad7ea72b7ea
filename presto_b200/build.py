"""Builds libaccel_b200.so in-tree for sm_100a (nvcc + gcc, no JIT cache).

The shared library holds the CUDA kernels, the device orchestration and the
host C code behind include/accel_b200.h.  It is written next to this file so
that it travels with the repository snapshot.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libaccel_b200.so")
# the reference's accel.h hot-path functions over the engine (include/accel_dropin.h)
DROPIN = os.path.join(HERE, "libaccel_dropin.so")
DROPIN_SRC = "accel_dropin.c"
BUILD = os.path.join(HERE, "_build")

CU_SOURCES = ["ab_kernels.cu", "ab_engine.cu", "ab_noalloc.cu", "ab_pool.cu", "ab_tc.cu", "ab_polish.cu", "ab_polish_rzw.cu", "ab_series.cu", "ab_dedisp.cu"]
C_SOURCES = ["ab_host.c", "ab_output.c", "ab_zap.c", "ab_dedisp.c"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-Xptxas", "-O3", "--expt-relaxed-constexpr"]
CC_FLAGS = ["-O2", "-g", "-fPIC", "-std=gnu11", "-pthread", "-ffp-contract=off", "-Wall",
            "-Wno-unused-function"]


def _cc():
    return "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return ([os.path.join(CSRC, s) for s in CU_SOURCES + C_SOURCES + [DROPIN_SRC]] +
            [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))] +
            [os.path.join(ROOT, "include", h) for h in os.listdir(os.path.join(ROOT, "include"))])


def up_to_date():
    if not os.path.exists(LIB) or not os.path.exists(DROPIN):
        return False
    t = min(os.path.getmtime(LIB), os.path.getmtime(DROPIN))
    return all(os.path.getmtime(s) <= t for s in sources())


def build_dropin():
    """libaccel_dropin.so: links libaccel_b200.so (found beside it at run
    time); glib's list functions and libpresto's free_accelcand stay
    undefined, resolved from the accelsearch process that loads it."""
    tmp = DROPIN + ".tmp"
    cmd = [_cc()] + CC_FLAGS + ["-shared", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
                                os.path.join(CSRC, DROPIN_SRC), "-o", tmp, "-L", HERE,
                                "-laccel_b200", "-Wl,-rpath,$ORIGIN", "-lm"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, DROPIN)
    return DROPIN


def build(force=False, verbose=False, ptxas_info=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    env = dict(os.environ)
    env.setdefault("CC", _cc())
    for s in C_SOURCES:
        o = os.path.join(BUILD, s + ".o")
        cmd = [_cc()] + CC_FLAGS + ["-I", os.path.join(ROOT, "include"), "-c",
                                    os.path.join(CSRC, s), "-o", o]
        subprocess.run(cmd, check=True)
        objs.append(o)
    for s in CU_SOURCES:
        o = os.path.join(BUILD, s + ".o")
        cmd = [_nvcc(), "-ccbin", "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"]
        cmd += NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_info else [])
        cmd += ["-I", os.path.join(ROOT, "include"), "-c", os.path.join(CSRC, s), "-o", o]
        r = subprocess.run(cmd, check=True, capture_output=True, text=True)
        if verbose or ptxas_info:
            sys.stderr.write(r.stdout + r.stderr)
        objs.append(o)
    tmp = LIB + ".tmp"
    cmd = [_nvcc(), "-ccbin", "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++",
           "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp] + objs + ["-lm", "-lpthread"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    build_dropin()
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
