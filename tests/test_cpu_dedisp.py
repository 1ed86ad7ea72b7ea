"""Subband dedispersion on the host: the product's integer delays equal those
prepsubband derives from the reference's own subband_search_delays /
subband_delays (src/dispersion.c compiled unmodified into
oracle/_ref/libref_dedisp.so), and the whole-array sums the device computes
(zero past the end of the data) equal the reference's dedisp_subbands and
float_dedisp streamed block by block as prepsubband streams them, bit for
bit.  The whole-array form is restated here in float32 numpy in the
reference's summation order."""
import numpy as np
import pytest

LO, BW, DT = 1200.0, 1.0, 1e-4


def _ref(oracle):
    L = oracle.ref_dedisp_lib()
    if L is None:
        pytest.skip("oracle/_ref/libref_dedisp.so is built where the reference tree is present")
    return L


def whole_array(X, cd, off, nsub, ds):
    nspec, nchan = X.shape
    cps = nchan // nsub
    Xp = np.concatenate([X, np.zeros((int(cd.max()) + 1, nchan), np.float32)])
    S = np.zeros((nsub, nspec), np.float32)
    for s in range(nsub):
        acc = np.zeros(nspec, np.float32)
        for j in range(cps):
            c = s * cps + j
            acc = (acc + Xp[cd[c]:cd[c] + nspec, c]).astype(np.float32)
        S[s] = acc
    nout = nspec // ds
    if ds > 1:
        ftmp = np.zeros((nsub, nout), np.float32)
        for k in range(ds):
            ftmp = (ftmp + S[:, k:nout * ds:ds]).astype(np.float32)
        D = (np.float32(0.0) + ftmp / np.float32(ds)).astype(np.float32)
    else:
        D = S[:, :nout]
    Dp = np.concatenate([D, np.zeros((nsub, int(off.max()) + 1), np.float32)], axis=1)
    out = np.zeros((off.shape[0], nout), np.float32)
    for d in range(off.shape[0]):
        acc = np.full(nout, -0.0, np.float32)
        for s in range(nsub):
            acc = (acc + Dp[s, off[d, s]:off[d, s] + nout]).astype(np.float32)
        out[d] = acc
    return out


@pytest.mark.parametrize("nchan,nsub,ds", [(64, 8, 1), (64, 16, 2), (96, 12, 4)])
def test_delays_match_reference(ablib, oracle, nchan, nsub, ds):
    L = _ref(oracle)
    dms = np.arange(0.0, 310.0, 7.5)
    cd, off = ablib.dedisp_delays(nchan, LO, BW, DT, nsub, dms, ds)
    rcd, roff = oracle.ref_dedisp_delays(L, nchan, LO, BW, DT, nsub, dms, ds)
    assert np.array_equal(cd, rcd) and np.array_equal(off, roff)
    assert cd.min() >= 0 and off.min() >= 0


@pytest.mark.parametrize("ds", [1, 2])
def test_whole_array_equals_streamed_reference(ablib, oracle, ds):
    L = _ref(oracle)
    rng = np.random.default_rng(ds)
    W, nb, nchan, nsub = 2048, 3, 32, 8
    X = rng.standard_normal((W * nb, nchan)).astype(np.float32)
    dms = np.arange(0.0, 120.0, 20.0)
    cd, off = ablib.dedisp_delays(nchan, LO, BW, DT, nsub, dms, ds)
    want = oracle.ref_dedisperse(L, X, LO, BW, DT, nsub, dms, ds, W)
    got = whole_array(X, cd, off, nsub, ds)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_delays_reject_descending_channels(ablib):
    with pytest.raises(ablib.AccelError):
        ablib.dedisp_delays(16, 1400.0, -1.0, DT, 4, [50.0], 1)
