"""The whole accelsearch run on the device (AccelSearch.run through the C ABI)
against the reference program's own output files (tests/golden/ref_accel/).

Per case (acceleration search in standard and in-memory mode, jerk search,
-locpow, -noharmpolish, -photon, and the benchmark configurations' search
parameters on N = 2^20 and, for the jerk search, N = 2^18), on the same
seeded spectrum (its SHA-256 checked):
* .txtcand: the same candidate insertions in the same order (numharm, r, z, w
  equal; power and sigma within the plane tolerance);
* .cand: the same candidates in the same order, r, z, w equal, the
  fourierprops fields within the tolerances of tests/ref_compare.py;
* the text file: both tables' title and rule lines and the appended .inf byte
  for byte, every row's fixed-width columns parsed and compared with the same
  tolerances.
"""
import hashlib
import os

import pytest

import ref_compare as rc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=sorted(rc.MANIFEST))
def run(request, ctx, ablib, tmp_path_factory):
    name = request.param
    case = rc.MANIFEST[name]
    mk = rc.maker()
    fft = mk.spectrum(case["N"], case["seed"], case["pulsars"])
    assert hashlib.sha256(fft.tobytes()).hexdigest() == case["fft_sha256"]
    tmp = tmp_path_factory.mktemp(name)
    root = str(tmp / name)
    with open(root + ".inf", "w") as f:
        f.write(mk.inf_text(name, case["N"], case["dt"]))
    kw = rc.opts(case["options"])
    if kw.get("photon"):
        kw["photon"] = float(fft[0].real)                # -photon: nph = fft[0].r
    s = ablib.AccelSearch(ctx=ctx, sigma=2.0, **kw)
    res = s.run(fft, case["N"], case["dt"], rootname=root)
    names = ablib.accel_filenames(root, res["obs"])
    mine = {k: open(v, "rb").read() for k, v in names.items()}
    assert sorted(os.path.basename(v) for v in names.values()) == sorted(case["files"])
    return dict(name=name, obs=res["obs"], mine=mine, gold=rc.gold_files(name))


def test_txtcand_matches_reference(run):
    rc.check_txtcand(run["name"], run["mine"]["txtcand"], run["gold"]["txtcand"])


def test_candfile_matches_reference(run, ablib):
    rc.check_candfile(run["name"], run["mine"]["cand"], run["gold"]["cand"], ablib.FourierProps)


def test_accelfile_matches_reference(run):
    rc.check_accelfile(run["name"], run["obs"].numw, run["mine"]["accel"], run["gold"]["accel"])
