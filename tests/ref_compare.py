"""Comparison of an accelsearch run's three output files with the reference
program's own (tests/golden/ref_accel/, made by tests/golden/make_ref_accel.py:
src/accelsearch.c and the libpresto files it links, compiled unmodified, with
FFTW / GSL / glib replaced by stand-ins written for this repository).

Tolerances.  The search is FP32 on both sides (the device's transforms
against an FP64-internal FFTW stand-in rounded to float): candidate lists,
their r, z, w and the columns derived from them (period, frequency, fdot,
acceleration, predicted harmonics, notes) agree exactly; summed powers and
sigmas to 1e-4.  Polishing maximises a flat peak whose objective carries
float rounding (epsilon ~ 1e-7) on both sides, so the two optimisers' maxima
agree only to ~sqrt(epsilon) ~ 3e-4 bins: phases and centroids to 5e-3,
purities (the power's second derivative) to 5 %, harmonic powers to 2e-3
relative + 2e-3 (powers are in units of the local noise power; noise-level
harmonics sit off their own maxima and move to first order), the coherent
sum of a candidate's harmonics to 5e-3 + 0.03.  Printed columns may also
round to neighbouring last digits.
"""
import hashlib
import importlib.util
import json
import os
import re

import numpy as np

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_accel")
MANIFEST = json.load(open(os.path.join(GOLD, "manifest.json")))


def maker():
    """tests/golden/make_ref_accel.py as a module (spectra, .inf text)."""
    spec = importlib.util.spec_from_file_location(
        "make_ref_accel", os.path.join(os.path.dirname(GOLD), "make_ref_accel.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def opts(options):
    """accelsearch options of a manifest case as AccelSearch keywords"""
    kw, it = {}, iter(options)
    for o in it:
        if o in ("-zmax", "-wmax", "-numharm"):
            kw[o[1:]] = int(next(it))
        elif o == "-locpow":
            kw["locpow"] = True
        elif o == "-noharmpolish":
            kw["noharmpolish"] = True
        elif o == "-photon":
            kw["photon"] = True          # the spectrum's DC term, set by the caller
        elif o == "-zaplist":
            next(it)                     # the case's zap list, written by the caller
        else:
            raise ValueError(o)
    return kw


def write_inputs(name, tmp):
    """the case's input files in tmp (<name>.fft or <name>.dat, .inf and any
    zap list); returns (input file name, the spectrum or series array)"""
    case = MANIFEST[name]
    mk = maker()
    if case.get("dat"):
        data = mk.series(case["N"], case["seed"], case["pulsars"])
        fname = name + ".dat"
    else:
        data = mk.spectrum(case["N"], case["seed"], case["pulsars"])
        fname = name + ".fft"
    assert hashlib.sha256(data.tobytes()).hexdigest() == case["fft_sha256"]
    data.tofile(os.path.join(tmp, fname))
    with open(os.path.join(tmp, name + ".inf"), "w") as f:
        f.write(mk.inf_text(name, case["N"], case["dt"]))
    if "zaplist" in case:
        with open(os.path.join(tmp, name + ".zaplist"), "w") as f:
            f.write(case["zaplist"])
    return fname, data


def gold_files(name):
    """{"accel" | "cand" | "txtcand": bytes} of the reference program's run"""
    gold = {}
    for f in MANIFEST[name]["files"]:
        k = "cand" if f.endswith(".cand") else "txtcand" if f.endswith(".txtcand") else "accel"
        gold[k] = open(os.path.join(GOLD, name, f), "rb").read()
    return gold


def _num(s):
    """(value, unit of its last printed digit) of a value(error)[x10^e] or a
    plain number column, or None when the column cut its exponent off (the
    reference's center_string truncates strings longer than the column)"""
    s = s.strip()
    m = re.match(r"^([-+]?)([0-9]*)(?:\.([0-9]*))?(?:e([-+]\d+))?", s)
    assert m and (m.group(2) or m.group(3)), s
    frac = m.group(3) or ""
    e = int(m.group(4) or 0)
    if "x10" in s:
        x = re.search(r"x10\^(-?\d+)$", s)
        if not x:
            return None
        e += int(x.group(1))
    v = float(m.group(1) + (m.group(2) or "0") + "." + (frac or "0")) * 10.0 ** e
    return v, 10.0 ** (e - len(frac))


def _cols(line, widths):
    out, p = [], 0
    for w in widths:
        out.append(line[p:p + w])
        p += w + 2
    return out, line[p:]


def _tables(text, numw):
    fw = [4, 5, 6, 8, 4, 16, 15, 15, 15, 11] + ([11] if numw else []) + [15]
    hw = [5, 4, 5, 15, 11, 18, 13, 12, 9] + ([12, 9] if numw else []) + [12, 10, 10]
    parts = text.split("\n\n\n")
    fund, harm, inf = parts[0], parts[1], "\n\n\n".join(parts[2:])
    fl, hl = fund.split("\n"), harm.split("\n")
    rows_f = [_cols(ln, fw) for ln in fl[3:]]
    rows_h = [_cols(ln, hw) for ln in hl[3:]]
    return fl[:3], rows_f, hl[:3], rows_h, inf


def close(a, b, rtol, atol=0.0):
    return abs(a - b) <= rtol * max(abs(a), abs(b)) + atol


def check_txtcand(name, mine, gold):
    mine = mine.decode().splitlines()
    gold = gold.decode().splitlines()
    assert len(mine) == len(gold), (name, len(mine), len(gold))
    for a, b in zip(mine, gold):
        fa, fb = a.split(), b.split()
        assert fa[2:] == fb[2:] or (fa[2] == fb[2] and all(
            close(float(x), float(y), 1e-9, 1e-4) for x, y in zip(fa[3:], fb[3:]))), (a, b)
        assert close(float(fa[0]), float(fb[0]), 1e-4, 0.011), (a, b)
        assert close(float(fa[1]), float(fb[1]), 1e-3, 1.1e-4), (a, b)


def check_candfile(name, mine, gold, FourierProps):
    import ctypes as C
    n = len(gold) // C.sizeof(FourierProps)
    assert len(mine) == len(gold), name
    mine = (FourierProps * n).from_buffer_copy(mine)
    gold = (FourierProps * n).from_buffer_copy(gold)
    for k, (a, b) in enumerate(zip(mine, gold)):
        info = (name, k)
        assert (a.r, a.z, a.w) == (b.r, b.z, b.w), info
        assert (a.rerr, a.zerr, a.werr) == (b.rerr, b.zerr, b.werr), info
        for f in ("pow", "powerr", "sig", "rawpow", "locpow", "phserr", "cenerr"):
            assert close(getattr(a, f), getattr(b, f), 2e-3, 2e-3), (info, f, getattr(a, f),
                                                                    getattr(b, f))
        assert abs(np.angle(np.exp(1j * (a.phs - b.phs)))) <= 5e-3, info
        assert abs(a.cen - b.cen) <= 5e-3, info
        for f in ("pur", "purerr"):
            assert close(getattr(a, f), getattr(b, f), 5e-2), (info, f, getattr(a, f),
                                                               getattr(b, f))


FUND_TOL = dict(sigma=(1e-4, 0), power=(1e-4, 0), coherent=(5e-3, 0.03), period=(1e-9, 0),
                freq=(1e-9, 0), r=(1e-9, 0), fdot=(1e-9, 0), z=(1e-9, 0), w=(1e-9, 0),
                accel=(1e-9, 0))
HARM_TOL = dict(sigma=(2e-3, 2e-3), pow=(2e-3, 2e-3), rawpow=(2e-3, 2e-3), r=(0, 1e-3),
                predr=(0, 0), z=(0, 1e-2), predz=(0, 0), w=(0, 0.1), predw=(0, 0),
                phase=(0, 5e-3), centroid=(0, 5e-3), purity=(5e-2, 0))


def _agree(sa, sb, rtol, atol, cut):
    """printed columns agree within rtol + atol + one unit of the last printed
    digit (the values may round to neighbouring digits).  A value(error)
    whose exponent the reference's center_string cut off can not be read (its
    digits are those of value / 10^e, e set by the error's own size); such
    cells are counted in cut[0] and skipped."""
    na, nb = _num(sa), _num(sb)
    if na is None or nb is None:
        cut[0] += 1
        return True
    (a, ua), (b, ub) = na, nb
    return abs(a - b) <= rtol * max(abs(a), abs(b)) + atol + 1.01 * max(ua, ub)


def check_accelfile(name, numw, mine, gold):
    fnames = ["cand", "sigma", "power", "coherent", "numharm", "period", "freq", "r", "fdot",
              "z"] + (["w"] if numw else []) + ["accel"]
    hnames = ["cand", "harm", "sigma", "pow", "rawpow", "r", "predr", "z", "predz"] + \
        (["w", "predw"] if numw else []) + ["phase", "centroid", "purity"]
    hf_a, rf_a, hh_a, rh_a, inf_a = _tables(mine.decode(), numw)
    hf_b, rf_b, hh_b, rh_b, inf_b = _tables(gold.decode(), numw)
    assert hf_a == hf_b and hh_a == hh_b and inf_a == inf_b
    assert len(rf_a) == len(rf_b) and len(rh_a) == len(rh_b), name
    cut, cells = [0], 0
    for (ca, na), (cb, nb) in zip(rf_a, rf_b):
        assert ca[0] == cb[0] and ca[4] == cb[4], (ca, cb)        # candidate, numharm
        assert na.rstrip() == nb.rstrip(), (na, nb)                # notes
        for k, col in enumerate(fnames):
            if col in FUND_TOL:
                cells += 1
                assert _agree(ca[k], cb[k], *FUND_TOL[col], cut), (name, col, ca[k], cb[k])
    for (ca, _), (cb, _) in zip(rh_a, rh_b):
        assert ca[0] == cb[0] and ca[1] == cb[1], (ca, cb)
        for k, col in enumerate(hnames):
            if col in HARM_TOL:
                cells += 1
                assert _agree(ca[k], cb[k], *HARM_TOL[col], cut), (name, col, ca[k], cb[k])
    assert cut[0] <= 0.02 * cells, (name, cut[0], cells)
