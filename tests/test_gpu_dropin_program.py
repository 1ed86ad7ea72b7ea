"""The reference's own accelsearch program on the B200 engine, through the
drop-in library that exports accel.h's hot-path functions
(libaccel_dropin.so, include/accel_dropin.h).

oracle/_ref/accelsearch_b200 is the unmodified src/accelsearch.c (with its
command-line parser and the libpresto files it links, as a shared
libpresto_ref.so over the FFTW/GSL/glib stand-ins) linked against
presto_b200/libaccel_dropin.so ahead of libpresto_ref.so: its main loop's
create_subharminfos / subharm_fderivs_vol / add_ffdotpows /
inmem_add_ffdotpows / fund_to_ffdotplane / search_ffdotpows calls bind to the
engine, everything else (create_accelobs, polishing, output) to the
reference's code.  Run on every golden case, its three output files must
match the reference program's own (tests/golden/ref_accel/) with the
tolerances of tests/ref_compare.py.  The stock dynamically linked program
(accelsearch_dyn) with the drop-in preloaded (LD_PRELOAD) must give the
same.  Both programs are built by oracle/build_ref.sh where the reference
tree is present.
"""
import os
import subprocess

import pytest

import ref_compare as rc

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROG = os.path.join(ROOT, "oracle", "_ref", "accelsearch_b200")
DYN = os.path.join(ROOT, "oracle", "_ref", "accelsearch_dyn")
DROPIN = os.path.join(ROOT, "presto_b200", "libaccel_dropin.so")


def _run_program(name, tmp, argv0, env=None):
    case = rc.MANIFEST[name]
    fname, _ = rc.write_inputs(name, tmp)
    r = subprocess.run([argv0] + case["options"] + [fname], cwd=tmp, capture_output=True,
                       text=True, timeout=1800, env=env)
    assert r.returncode == 0, (name, r.stdout[-3000:], r.stderr[-3000:])
    assert "on the GPU" in r.stdout, "the drop-in's create_subharminfos did not run"
    mine = {}
    for f in case["files"]:
        k = "cand" if f.endswith(".cand") else "txtcand" if f.endswith(".txtcand") else "accel"
        mine[k] = open(os.path.join(tmp, f), "rb").read()
    return mine


def _check(name, mine, ablib):
    gold = rc.gold_files(name)
    numw = 1 if "-wmax" in rc.MANIFEST[name]["options"] and \
        int(rc.MANIFEST[name]["options"][rc.MANIFEST[name]["options"].index("-wmax") + 1]) else 0
    if "txtcand" in gold:
        rc.check_txtcand(name, mine["txtcand"], gold["txtcand"])
    rc.check_candfile(name, mine["cand"], gold["cand"], ablib.FourierProps)
    rc.check_accelfile(name, numw, mine["accel"], gold["accel"])


@pytest.mark.parametrize("name", sorted(rc.MANIFEST))
def test_reference_program_on_dropin(name, ablib, tmp_path):
    if not os.path.exists(PROG):
        pytest.skip("oracle/_ref/accelsearch_b200 is built where the reference tree is present")
    _check(name, _run_program(name, str(tmp_path), PROG), ablib)


@pytest.mark.parametrize("name", ["jerk", "inmem"])
def test_stock_program_with_preloaded_dropin(name, ablib, tmp_path):
    if not os.path.exists(DYN):
        pytest.skip("oracle/_ref/accelsearch_dyn is built where the reference tree is present")
    env = dict(os.environ, LD_PRELOAD=DROPIN)
    _check(name, _run_program(name, str(tmp_path), DYN, env=env), ablib)
