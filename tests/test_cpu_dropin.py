"""libaccel_dropin.so on the CPU: it loads, exports exactly the accel.h
functions include/accel_dropin.h declares, its structures have the
reference's member offsets, and the reference program linked against it
binds the main loop's hot-path calls to it and the rest to libpresto."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "include", "accel_dropin.h")
LIB = os.path.join(ROOT, "presto_b200", "libaccel_dropin.so")
REF_LAYOUT = os.path.join(ROOT, "oracle", "_ref", "accel_layout.txt")
PROG = os.path.join(ROOT, "oracle", "_ref", "accelsearch_b200")
CC = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"


def _declared():
    text = open(HDR).read()
    return set(re.findall(r"^\w[\w\s\*]*?\b(\w+)\s*\(", text, re.M))


def test_exports_every_declared_function(ablib):
    import ctypes as C
    names = _declared()
    assert names == {"create_subharminfos", "free_subharminfos", "subharm_fderivs_vol",
                     "copy_ffdotpows", "fund_to_ffdotplane", "inmem_add_ffdotpows",
                     "fund_to_ffdotplane_trans", "inmem_add_ffdotpows_trans", "free_ffdotpows",
                     "add_ffdotpows_ptrs", "add_ffdotpows", "search_ffdotpows"}
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True,
                         check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert names <= exported, names - exported
    # only glib's list calls and libpresto's accelcand destructor are left to
    # the loading process
    out = subprocess.run(["nm", "-D", "--undefined-only", LIB], capture_output=True, text=True,
                         check=True).stdout
    # (C library symbols carry a version, the engine's are ab_*)
    undef = {ln.split()[-1] for ln in out.splitlines() if ln.split()[0] == "U"}
    foreign = {u for u in undef if "@" not in u and not u.startswith("ab_")}
    assert foreign == {"g_slist_alloc", "g_slist_remove_link", "g_slist_free_1",
                       "free_accelcand"}, foreign
    C.CDLL(os.path.join(ROOT, "presto_b200", "libaccel_b200.so"))
    C.CDLL(LIB, mode=os.RTLD_LAZY)           # glib and libpresto come from the program


def test_structures_match_the_reference_layout(tmp_path):
    if not os.path.exists(REF_LAYOUT):
        pytest.skip("oracle/_ref/accel_layout.txt is written where the reference tree is present")
    exe = str(tmp_path / "probe")
    subprocess.run([CC, "-DDROPIN", "-I", os.path.join(ROOT, "include"), "-o", exe,
                    os.path.join(ROOT, "oracle", "layout_probe.c")], check=True)
    mine = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    assert mine == open(REF_LAYOUT).read()


def test_reference_program_binds_the_hot_path_to_the_dropin(tmp_path):
    if not os.path.exists(PROG):
        pytest.skip("oracle/_ref/accelsearch_b200 is built where the reference tree is present")
    env = dict(os.environ, LD_DEBUG="bindings", LD_BIND_NOW="1")
    r = subprocess.run([PROG], capture_output=True, text=True, env=env, cwd=str(tmp_path))
    binds = {}
    for ln in r.stderr.splitlines():
        m = re.search(r"binding file \S+accelsearch_b200 \[0\] to (\S+) \[0\]: normal symbol "
                      r"`(\w+)'", ln)
        if m:
            binds[m.group(2)] = os.path.basename(m.group(1))
    for f in ("create_subharminfos", "subharm_fderivs_vol", "search_ffdotpows", "add_ffdotpows",
              "free_ffdotpows", "free_subharminfos"):
        assert binds.get(f) == "libaccel_dropin.so", (f, binds.get(f))
    for f in ("create_accelobs", "optimize_accelcand", "output_fundamentals"):
        assert binds.get(f) == "libpresto_ref.so", (f, binds.get(f))
