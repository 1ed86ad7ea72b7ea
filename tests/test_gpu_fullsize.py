"""Parity at the benchmark searches' full lengths, through the C ABI.

The two large searches are checked at their real sizes, not only through
their parameters on shorter spectra:

* the jerk search (N = 2^22, zmax = 200, wmax = 300, numharm = 8: 31 w planes
  x 201 z rows at the fundamental, seven subharmonic banks up to 177 x 27),
  which exercises calc_required_w / index_from_w and the w field of the hit
  key at numw = 31 (src/accel_utils.c:54-102, 1261-1309);
* the larger acceleration search (N = 2^23, zmax = 600, numharm = 16) on its
  last blocks: high block ordinals, the last superblock groups and the last
  partial batch of a search of ~3090 blocks.

Each check runs the whole device search (every block, so the blocks under test
sit in the batches, superblocks and hit ring of a real search) and compares
the threshold crossings of a window of blocks with the oracle's search of
that window (src/accel_utils.c:1412-1452), then compares a windowed device
search's candidate list with the oracle's list for the same window
(insert_new_accelcand order, src/accel_utils.c:387-469).  Planes of the
jerk search's fundamental and widest subharmonic bank are compared cell for
cell.  Tolerances are those of tests/test_gpu_parity.py: powers within 1e-4
relative, hit keys identical apart from crossings within 1e-4 of the power
cut, candidates with identical numharm and r, z, w within 1e-3 bins.
"""
import os

import numpy as np
import pytest

from presto_b200 import synth

pytestmark = pytest.mark.gpu
DT = 64e-6
PTOL = 1e-4
NTHREADS = os.cpu_count() or 1


def _borderline(pw, stage, obs):
    return abs(pw - obs.powcut[stage]) <= 1e-4 * obs.powcut[stage]


def _hit_dict(blk, st, wi, zi, ri, pw, lo, hi):
    sel = (blk >= lo) & (blk < hi)
    return {(int(b), int(s), int(w), int(z), int(r)): float(p)
            for b, s, w, z, r, p in zip(blk[sel], st[sel], wi[sel], zi[sel], ri[sel], pw[sel])}


def _compare_hits(dset, ohits, obs):
    oset = {(b, s, w, z, r): p for b, s, w, z, r, p in ohits}
    only_d = [k for k in dset if k not in oset and not _borderline(dset[k], k[1], obs)]
    only_o = [k for k in oset if k not in dset and not _borderline(oset[k], k[1], obs)]
    assert not only_d and not only_o, (len(only_d), len(only_o), only_d[:5], only_o[:5])
    for k in set(dset) & set(oset):
        assert abs(dset[k] - oset[k]) <= PTOL * oset[k], (k, dset[k], oset[k])
    return len(oset)


def _compare_cands(dev, ocands):
    assert len(dev) == len(ocands), (len(dev), len(ocands))
    for d, o in zip(dev, ocands):
        assert d[2] == o[2], (d, o)
        assert abs(d[3] - o[3]) < 1e-3 and abs(d[4] - o[4]) < 1e-3 and abs(d[5] - o[5]) < 1e-3
        assert abs(d[0] - o[0]) <= PTOL * o[0], (d, o)
        assert abs(d[1] - o[1]) <= 1e-3 * max(o[1], 1.0), (d, o)


def _close(dev, orc):
    tol = PTOL * (orc + max(float(orc.mean()), 1e-3))
    return bool(np.all(np.abs(dev - orc) <= tol)), float(np.max(np.abs(dev - orc) / (orc + 1.0)))


class _Search:
    def __init__(self, ablib, oracle, N, fft, **kw):
        self.N, self.fft, self.kw = N, fft, kw
        self.obs = ablib.obs_init(ablib.make_params(N, DT, fft.size, **kw))
        self.p = oracle.make_params(N, DT, fft.size, **kw)
        self.oobs = oracle.obs_init(self.p)
        self.nblocks = ablib.num_blocks(self.obs)


@pytest.fixture(scope="module")
def jerk(ablib, oracle, ctx):
    fft, _ = synth.cfg3_spectrum(N=1 << 22, dt=DT, seed=3000)
    s = _Search(ablib, oracle, 1 << 22, fft, zmax=200, wmax=300, numharm=8)
    assert (s.obs.numz, s.obs.numw, s.obs.numharmstages) == (201, 31, 4)
    ctx.search(s.obs, fft)
    s.hits = ctx.last_hits()
    return s


@pytest.fixture(scope="module")
def accel(ablib, oracle, ctx):
    fft, _ = synth.cfg2_spectrum(N=1 << 23, dt=DT, seed=2000)
    s = _Search(ablib, oracle, 1 << 23, fft, zmax=600, numharm=16)
    assert (s.obs.numz, s.obs.numharmstages, s.obs.inmem) == (601, 5, 0)
    ctx.search(s.obs, fft)
    s.hits = ctx.last_hits()
    return s


def _window(ctx, oracle, s, first, count, expect_hits):
    ocands, ohits, nb = oracle.accelsearch(s.p, s.fft, nthreads=NTHREADS, first_block=first,
                                           max_blocks=count, maxhits=4000000)
    assert nb == count and len(ohits) < 4000000
    n = _compare_hits(_hit_dict(*s.hits, first, first + count), ohits, s.obs)
    if expect_hits:
        assert n > 0, "the window must hold threshold crossings"
    dev = ctx.search(s.obs, s.fft, first_block=first, max_blocks=count)
    _compare_cands(dev, ocands)


def test_jerk_hits_near_injection(ctx, oracle, jerk):
    """Blocks 4-11 hold the fundamental of the injected sinusoid at r ~ 5880
    (z ~ -42, w ~ -61) and the jerk planes its harmonics smear into."""
    _window(ctx, oracle, jerk, 4, 8, True)


def test_jerk_hits_mid_spectrum(ctx, oracle, jerk):
    """Noise only: no crossings on either side."""
    _window(ctx, oracle, jerk, jerk.nblocks // 2, 8, False)


def test_jerk_hits_highest_crossings(ctx, oracle, jerk):
    """The 8 blocks ending at the highest block with a crossing in the whole
    device search."""
    top = int(jerk.hits[0].max())
    _window(ctx, oracle, jerk, max(0, top - 7), 8, True)


def test_jerk_key_fields(jerk):
    """The hit keys span the whole jerk grid: w indices up to numw-1 = 30 and
    every harmonic stage."""
    blk, st, wi, zi, ri, pw = jerk.hits
    assert len(blk) > 0
    assert int(wi.max()) == jerk.obs.numw - 1 and int(wi.min()) == 0
    assert int(zi.max()) <= jerk.obs.numz - 1
    assert set(np.unique(st).tolist()) == set(range(jerk.obs.numharmstages))


@pytest.mark.parametrize("nh,hn", [(1, 1), (8, 7), (2, 1)])
def test_jerk_planes(ctx, oracle, jerk, nh, hn):
    """The fundamental (201 x 31 templates), the widest subharmonic bank (7/8:
    177 x 27) and the 1/2 bank, cell for cell, on a low block and a high one."""
    ctx.set_spectrum(jerk.obs, jerk.fft)
    bank = oracle.Bank(jerk.oobs, nh, hn)
    for b in (6, jerk.nblocks - 3):
        lo = jerk.obs.rlo + b * jerk.obs.rstep
        hi = lo + jerk.obs.rstep - 0.5
        meta, dev = ctx.subharm_fderivs_vol(jerk.obs, nh, hn, lo, hi)
        ometa, orc, _, _ = oracle.subharm_fderivs_vol(jerk.oobs, jerk.fft, nh, hn, lo, hi, bank)
        assert meta == ometa, (b, meta, ometa)
        ok, worst = _close(dev, orc)
        assert ok, (nh, hn, b, worst)


def test_accel_last_blocks(ctx, oracle, accel):
    """The last 16 blocks of the N = 2^23 search (the top of the spectrum, the
    last superblock groups and batch): noise only, no crossings on either
    side."""
    _window(ctx, oracle, accel, accel.nblocks - 16, 16, False)


def test_accel_highest_crossings(ctx, oracle, accel):
    """The 16 blocks ending at the highest block with a crossing in the whole
    device search (a pulsar harmonic far up the spectrum)."""
    top = int(accel.hits[0].max())
    _window(ctx, oracle, accel, max(0, top - 15), 16, True)


def test_accel_high_block_planes(ctx, oracle, accel):
    """The fundamental and the 15/16 bank's planes at the highest block."""
    ctx.set_spectrum(accel.obs, accel.fft)
    b = accel.nblocks - 1
    lo = accel.obs.rlo + b * accel.obs.rstep
    hi = lo + accel.obs.rstep - 0.5
    for nh, hn in ((1, 1), (16, 15)):
        bank = oracle.Bank(accel.oobs, nh, hn)
        meta, dev = ctx.subharm_fderivs_vol(accel.obs, nh, hn, lo, hi)
        ometa, orc, _, _ = oracle.subharm_fderivs_vol(accel.oobs, accel.fft, nh, hn, lo, hi, bank)
        assert meta == ometa
        ok, worst = _close(dev, orc)
        assert ok, (nh, hn, worst)
