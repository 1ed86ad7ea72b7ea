"""The whole accelsearch run on the device (AccelSearch.run through the C ABI)
against the reference program's own output files (tests/golden/ref_accel/).

Per case (acceleration search in standard and in-memory mode, jerk search,
-locpow, -noharmpolish, -photon, and the benchmark configurations' search
parameters on N = 2^20 and, for the jerk search, N = 2^18, and a .dat time
series with a zap list, searched through the device's realfft, deredden and
zapping), on the same seeded input (its SHA-256 checked):
* .txtcand: the same candidate insertions in the same order (numharm, r, z, w
  equal; power and sigma within the plane tolerance);
* .cand: the same candidates in the same order, r, z, w equal, the
  fourierprops fields within the tolerances of tests/ref_compare.py;
* the text file: both tables' title and rule lines and the appended .inf byte
  for byte, every row's fixed-width columns parsed and compared with the same
  tolerances.
"""
import os

import pytest

import ref_compare as rc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=sorted(rc.MANIFEST))
def run(request, ctx, ablib, tmp_path_factory):
    name = request.param
    case = rc.MANIFEST[name]
    tmp = tmp_path_factory.mktemp(name)
    root = str(tmp / name)
    _, data = rc.write_inputs(name, str(tmp))
    kw = rc.opts(case["options"])
    if kw.get("photon"):
        kw["photon"] = float(data[0].real)               # -photon: nph = fft[0].r
    s = ablib.AccelSearch(ctx=ctx, sigma=2.0, **kw)
    if case.get("dat"):
        # realfft + deredden on the device, the zap list applied to the
        # device spectrum
        zap = root + ".zaplist" if "zaplist" in case else None
        res = s.run_series(data, case["dt"], zaplist=zap, rootname=root)
    else:
        res = s.run(data, case["N"], case["dt"], rootname=root)
    names = ablib.accel_filenames(root, res["obs"])
    mine = {k: open(v, "rb").read() for k, v in names.items() if os.path.exists(v)}
    assert sorted(os.path.basename(names[k]) for k in mine) == sorted(case["files"])
    return dict(name=name, obs=res["obs"], mine=mine, gold=rc.gold_files(name))


def test_txtcand_matches_reference(run):
    if "txtcand" not in run["gold"]:
        pytest.skip("a .dat search writes no .txtcand")
    rc.check_txtcand(run["name"], run["mine"]["txtcand"], run["gold"]["txtcand"])


def test_candfile_matches_reference(run, ablib):
    rc.check_candfile(run["name"], run["mine"]["cand"], run["gold"]["cand"], ablib.FourierProps)


def test_accelfile_matches_reference(run):
    rc.check_accelfile(run["name"], run["obs"].numw, run["mine"]["accel"], run["gold"]["accel"])
