"""The parallel replay of a batch of threshold crossings
(ab_list_replay_parallel: clusters of r replayed on several threads; and
ab_replay_hits, which sorts a batch with re-packed keys and fills the
candidate fields on several threads before it) leaves the candidate list and
the .txtcand work-file text exactly as replaying the crossings one by one
through ab_list_insert (insert_new_accelcand, src/accel_utils.c:387-469)
does.  Host code only."""
import ctypes as C

import numpy as np
import pytest

import presto_b200 as pb


class Cand(C.Structure):
    _fields_ = [("power", C.c_float), ("sigma", C.c_float), ("numharm", C.c_int),
                ("r", C.c_double), ("z", C.c_double), ("w", C.c_double)]


@pytest.fixture(scope="module")
def L():
    L = pb.lib()
    vp, ll = C.c_void_p, C.c_longlong
    L.ab_list_new.restype = vp
    L.ab_list_free.argtypes = [vp]
    L.ab_list_insert.argtypes = [vp, C.c_float, C.c_float, C.c_int, C.c_double, C.c_double,
                                 C.c_double]
    L.ab_list_get.argtypes = [vp, vp, ll]
    L.ab_list_get.restype = ll
    L.ab_list_worklog.argtypes = [vp, C.c_int, C.c_double]
    L.ab_list_worklog_text.argtypes = [vp, C.POINTER(C.c_size_t)]
    L.ab_list_worklog_text.restype = C.c_void_p
    L.ab_list_replay_parallel.argtypes = [vp, ll, vp, vp, vp, vp, vp, vp, C.c_int]
    return L


def _new(L):
    l = L.ab_list_new()
    L.ab_list_worklog(l, 1, 67.1)
    return l


def _serial(L, l, h):
    for i in range(h["n"]):
        assert L.ab_list_insert(l, float(h["pw"][i]), float(h["sg"][i]), int(h["nh"][i]),
                                float(h["rr"][i]), float(h["zz"][i]), float(h["ww"][i])) >= 0


def _parallel(L, l, h, nt):
    a = [np.ascontiguousarray(h[k]) for k in ("pw", "sg", "nh", "rr", "zz", "ww")]
    rc = L.ab_list_replay_parallel(l, h["n"], *[x.ctypes.data for x in a], nt)
    assert rc == 0, rc


def _state(L, l):
    n = L.ab_list_get(l, None, 0)
    arr = (Cand * max(n, 1))()
    L.ab_list_get(l, arr, n)
    cands = [(c.power, c.sigma, c.numharm, c.r, c.z, c.w) for c in arr[:n]]
    ln = C.c_size_t()
    p = L.ab_list_worklog_text(l, C.byref(ln))
    return cands, C.string_at(p, ln.value)


def _batch(rng, n, centres, width, r_scale=0.5):
    """Crossings around the given r centres, in a random (visit) order, with
    r on the half-bin grid divided by the harmonic count as the search makes
    them."""
    nh = rng.choice([1, 2, 4, 8], size=n).astype(np.int32)
    c = rng.choice(centres, size=n)
    rr = (np.round((c * nh + rng.uniform(-width, width, n) * nh) / r_scale) * r_scale) / nh
    return dict(n=n, pw=rng.uniform(5, 60, n).astype(np.float32),
                sg=rng.uniform(2, 9, n).astype(np.float32), nh=nh, rr=rr.astype(np.float64),
                zz=rng.uniform(-200, 200, n), ww=np.zeros(n))


@pytest.mark.parametrize("seed", range(12))
@pytest.mark.parametrize("nt", [1, 3, 8])
def test_parallel_replay_equals_serial(L, seed, nt):
    rng = np.random.default_rng(seed)
    # an earlier batch builds the list (including nodes the tail rules put out
    # of order), then a dense batch: clusters below the list's last node, at
    # it, and several above it whose first crossings interleave
    old = np.sort(rng.uniform(50, 4000, 12))
    prev = _batch(rng, 3000, old, 40.0)
    new_centres = np.concatenate([old[rng.choice(old.size, 5, replace=False)],
                                  rng.uniform(4100, 9000, 6)])
    cur = _batch(rng, 20000, new_centres, 25.0 + 10 * (seed % 3))
    a, b = _new(L), _new(L)
    try:
        _serial(L, a, prev)
        _serial(L, b, prev)
        before = _state(L, b)
        _serial(L, a, cur)
        _parallel(L, b, cur, nt)
        sa, sb = _state(L, a), _state(L, b)
        assert sa[0] == sb[0]
        assert sa[1] == sb[1]
        assert len(sa[1]) > len(before[1])
    finally:
        L.ab_list_free(a)
        L.ab_list_free(b)


def test_parallel_replay_into_empty_list_with_tail_handover(L):
    """Every cluster new: each one's tail rules hold only until a higher
    cluster's first crossing arrives, and crossings alternate between clusters
    15 bins apart and closer."""
    rng = np.random.default_rng(99)
    centres = np.array([100.0, 116.0, 131.5, 400.0, 415.0, 1000.0])
    cur = _batch(rng, 30000, centres, 6.0)
    a, b = _new(L), _new(L)
    try:
        _serial(L, a, cur)
        _parallel(L, b, cur, 6)
        assert _state(L, a) == _state(L, b)
    finally:
        L.ab_list_free(a)
        L.ab_list_free(b)


def _keys(rng, n, nblocks, numz, numr, stages):
    blk = rng.integers(0, nblocks, n).astype(np.uint64)
    st = rng.integers(0, stages, n).astype(np.uint64)
    # crossings bunched around a few r and z cells, as a signal's harmonics give
    rc = rng.choice(rng.integers(0, numr, 8), n)
    r = np.clip(rc + rng.integers(-40, 41, n), 0, numr - 1).astype(np.uint64)
    z = np.clip(rng.choice(rng.integers(0, numz, 5), n) + rng.integers(-20, 21, n), 0,
                numz - 1).astype(np.uint64)
    k = (blk << np.uint64(38)) | (st << np.uint64(35)) | (z << np.uint64(16)) | r
    return np.unique(k)          # one crossing per (block, stage, w, z, r) cell


def test_replay_hits_batch_equals_serial_chunks(L):
    """ab_replay_hits on one large batch (sorted with re-packed keys, fields on
    several threads, clusters replayed in parallel) against the same crossings
    sorted and fed in chunks small enough for the one-by-one path: the same
    list, work-file text, and sorted keys, powers and sigmas."""
    obs = pb.obs_init(pb.make_params(1 << 20, 64e-6, 1 << 19, zmax=200, numharm=8, sigma=2.0))
    L.ab_replay_hits.argtypes = [C.POINTER(type(obs)), C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_longlong, C.c_void_p, C.c_longlong, C.c_void_p]
    rng = np.random.default_rng(7)
    keys = _keys(rng, 200000, 60, obs.numz, obs.corr_uselen, 4)
    n = keys.size
    perm = rng.permutation(n)
    pw = rng.uniform(5, 60, n).astype(np.float32)
    sg = rng.uniform(2, 9, n).astype(np.float32)
    startr = np.ascontiguousarray(obs.rlo + np.arange(700) * obs.rstep, dtype=np.float64)
    a, b = _new(L), _new(L)
    try:
        ka, pa, sa = (np.ascontiguousarray(x[perm]) for x in (keys, pw, sg))
        assert L.ab_replay_hits(C.byref(obs), ka.ctypes.data, pa.ctypes.data, sa.ctypes.data,
                                n, startr.ctypes.data, 700, a) == 0
        order = np.argsort(keys, kind="stable")
        kb, pb_, sb = (np.ascontiguousarray(x[order]) for x in (keys, pw, sg))
        for lo in range(0, n, 30000):
            hi = min(n, lo + 30000)
            k1, p1, s1 = kb[lo:hi].copy(), pb_[lo:hi].copy(), sb[lo:hi].copy()
            assert L.ab_replay_hits(C.byref(obs), k1.ctypes.data, p1.ctypes.data, s1.ctypes.data,
                                    hi - lo, startr.ctypes.data, 700, b) == 0
        assert np.array_equal(ka, kb) and np.array_equal(pa, pb_) and np.array_equal(sa, sb)
        sa_, sb_ = _state(L, a), _state(L, b)
        assert sa_[0] == sb_[0] and sa_[1] == sb_[1] and len(sa_[0]) > 5
    finally:
        L.ab_list_free(a)
        L.ab_list_free(b)


def test_parallel_replay_many_sparse_clusters(L):
    """Thousands of clusters (scattered noise crossings over a long r range),
    most of the list's candidates untouched by the batch."""
    rng = np.random.default_rng(5)
    prev = _batch(rng, 20000, rng.uniform(100, 2e6, 8000), 3.0)
    cur = _batch(rng, 40000, rng.uniform(100, 2.2e6, 6000), 3.0)
    a, b = _new(L), _new(L)
    try:
        _serial(L, a, prev)
        _serial(L, b, prev)
        _serial(L, a, cur)
        _parallel(L, b, cur, 8)
        sa, sb = _state(L, a), _state(L, b)
        assert sa == sb and len(sa[0]) > 5000
    finally:
        L.ab_list_free(a)
        L.ab_list_free(b)
