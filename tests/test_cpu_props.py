"""Candidate properties and the .cand file (host C in libaccel_b200.so):
ab_calc_props / ab_calc_rzwerrs against the oracle's restatements of
calc_props and calc_rzwerrs (src/characteristics.c:195-264, 353-392) bit for
bit, the reference's exit conditions as errors, the .cand records of
src/accelsearch.c:261-272 and the binary layout of fourierprops
(include/presto.h:170-188) that the .cand file is an array of."""
import ctypes as C

import numpy as np
import pytest

import presto_b200 as pb


def _random_derivs(rng, n):
    out = []
    for _ in range(n):
        locpow = float(rng.uniform(0.2, 5.0))
        powr = float(rng.uniform(5.0, 5e4)) * locpow
        out.append([powr, float(rng.uniform(0, 2 * np.pi)), float(rng.normal(0, 50)),
                    float(rng.normal(0, 3)), -float(rng.uniform(0.1, 4.0)) * powr,
                    float(rng.normal(0, 30)), locpow])
    return out


def _fields(s):
    return [getattr(s, f[0]) for f in s._fields_]


def test_calc_props_matches_oracle_bit_for_bit(oracle):
    L = oracle._polish_lib()
    rng = np.random.default_rng(31)
    for d in _random_derivs(rng, 400):
        r, z, w = float(rng.uniform(10, 1e6)), float(rng.normal(0, 100)), float(rng.normal(0, 300))
        mine = pb.calc_props(d, r, z, w)
        ref = oracle.FourierProps()
        assert L.orc_calc_props(oracle.RDerivs(*d), r, z, w, C.byref(ref)) == 0
        assert _fields(mine) == _fields(ref), (d, _fields(mine), _fields(ref))


def test_calc_rzwerrs_matches_oracle_bit_for_bit(oracle):
    L = oracle._polish_lib()
    L.orc_calc_rzwerrs.argtypes = [C.c_void_p, C.c_double, C.c_void_p]
    rng = np.random.default_rng(32)
    for d in _random_derivs(rng, 200):
        for w in (0.0, float(rng.normal(0, 300))):
            props = pb.calc_props(d, float(rng.uniform(10, 1e6)), float(rng.normal(0, 100)), w)
            T = float(rng.uniform(10, 2000))
            mine = pb.calc_rzwerrs(props, T)
            ref = pb.RzwErrs()
            assert L.orc_calc_rzwerrs(C.addressof(props), T, C.addressof(ref)) == 0
            assert _fields(mine) == _fields(ref)
            assert mine.pdd == 0.0 if w == 0.0 else True


def test_reference_exit_conditions_are_errors():
    with pytest.raises(pb.AccelError):
        pb.calc_props([1e-15, 0, 0, 0, 0, 0, 1.0], 10.0, 0.0, 0.0)
    with pytest.raises(pb.AccelError):
        pb.calc_props([10.0, 0, 0, 0, -1.0, 0, 1e-15], 10.0, 0.0, 0.0)
    props = pb.calc_props([10.0, 0, 0, 0, -1.0, 0, 1.0], 10.0, 0.0, 0.0)
    with pytest.raises(pb.AccelError):
        pb.calc_rzwerrs(props, 0.0)


def test_pure_tone_has_unit_purity():
    """|X(r0 + d)|^2 = P sinc^2(d) has d2P/dr2 = -2 pi^2 P / 3 at the peak,
    which calc_props maps to purity 1 (a signal present for the whole run)."""
    P = 1.0e4
    props = pb.calc_props([P, 0.3, 0.0, 0.0, -2.0 * np.pi ** 2 * P / 3.0, 0.0, 1.0], 500.0, 0.0, 0.0)
    assert abs(props.pur - 1.0) < 1e-6
    assert abs(props.pow - P) < 1e-3 and abs(props.powerr - np.sqrt(2 * P)) < 1e-3
    assert abs(props.rerr - 3.0 / (np.pi * np.sqrt(6 * P))) < 1e-7


def test_cand_file_records_and_layout(tmp_path):
    """src/accelsearch.c:261-272: calc_props of the fundamental's derivs at
    the search's (r, z, w), errors overridden by ACCEL_DR/DZ/DW / numharm;
    the file is the raw struct array (88 bytes per record on LP64)."""
    rng = np.random.default_rng(33)
    cands, pol = [], []
    for k, nh in enumerate((1, 2, 4, 8, 16)):
        cands.append((50.0 + k, 6.0 + k, nh, 1000.5 + 97 * k, 3.0 * k, 20.0 * k))
        pol.append(dict(pows=np.zeros(nh), derivs=np.array(_random_derivs(rng, nh))))
    props = pb.cand_props(cands, pol)
    for c, p, pr in zip(cands, pol, props):
        ref = pb.calc_props(p["derivs"][0], c[3], c[4], c[5])
        nh = c[2]
        assert (pr.r, pr.z, pr.w) == (c[3], c[4], c[5])
        assert pr.rerr == np.float32(0.5) / np.float32(nh)
        assert pr.zerr == np.float32(2.0) / np.float32(nh)
        assert pr.werr == np.float32(20.0) / np.float32(nh)
        assert (pr.pow, pr.sig, pr.phs, pr.pur, pr.locpow) == (ref.pow, ref.sig, ref.phs, ref.pur,
                                                                ref.locpow)
    assert C.sizeof(pb.FourierProps) == 88
    offs = {f[0]: getattr(pb.FourierProps, f[0]).offset for f in pb.FourierProps._fields_}
    assert (offs["r"], offs["rerr"], offs["z"], offs["zerr"], offs["w"], offs["werr"]) == \
        (0, 8, 16, 24, 32, 40)
    assert offs["pow"] == 44 and offs["locpow"] == 84
    path = tmp_path / "x_ACCEL_200.cand"
    pb.write_candfile(str(path), props)
    assert path.stat().st_size == 88 * len(props)
    back = pb.read_candfile(str(path))
    assert [_fields(a) for a in back] == [_fields(b) for b in props]
