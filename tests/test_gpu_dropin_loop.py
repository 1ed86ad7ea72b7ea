"""The reference's main search loop (src/accelsearch.c:186-214) driven through
the per-block drop-in entry points, as a maintainer binding the reference
driver to the C ABI would run it: per block subharm_fderivs_vol of the
fundamental, search_ffdotpows, then per stage subharm_fderivs_vol +
add_ffdotpows of each odd harmonic and search_ffdotpows, into one candidate
list with the .txtcand log on.  Against the whole-spectrum ab_search of the
same spectrum: the same candidates (numharm, r, z, w equal; power and sigma
within the plane tolerance, 1e-4) and the same .txtcand insertions in order.
Standard mode (the drop-in add_ffdotpows path; in-memory searches use
fund_to_ffdotplane + inmem_add_ffdotpows, checked in test_gpu_parity.py)."""
import numpy as np
import pytest

from presto_b200 import synth

pytestmark = pytest.mark.gpu
DT = 64e-6


def _close(a, b, rtol):
    return abs(a - b) <= rtol * max(abs(a), abs(b)) + 1e-6


def test_dropin_loop_matches_ab_search(ctx, ablib):
    N = 1 << 17
    fft = synth.spectrum(synth.time_series(N, 21, [dict(r=2100.4, z=-14.0, harms=[(0.07, 0.2),
                                                                                (0.05, 0.8),
                                                                                (0.04, 1.9)])]))
    obs = ablib.obs_init(ablib.make_params(N, DT, fft.size, zmax=40, wmax=0, numharm=4))
    assert not obs.inmem and obs.numharmstages == 3
    lst = ablib.CandList()
    lst.set_worklog(True, obs.T)
    ctx.set_spectrum(obs, fft)
    startr = obs.rlo
    nblocks = 0
    while startr + obs.rstep < obs.highestbin:
        nextr = startr + obs.rstep
        lastr = nextr - 0.5
        fmeta, fund = ctx.subharm_fderivs_vol(obs, 1, 1, startr, lastr)
        ctx.search_ffdotpows(obs, fmeta, fund, 1, lst)
        for stage in range(1, obs.numharmstages):
            h2s = 1 << stage
            for harm in range(1, h2s, 2):
                smeta, sub = ctx.subharm_fderivs_vol(obs, h2s, harm, startr, lastr)
                fund = ctx.add_ffdotpows(obs, fmeta, fund, smeta, sub, h2s, harm, startr)
            ctx.search_ffdotpows(obs, fmeta, fund, h2s, lst)
        startr = nextr
        nblocks += 1
    assert nblocks > 20
    loop_cands, loop_log = lst.get(), lst.worklog().splitlines()

    ctx.set_worklog(True)
    try:
        cands = ctx.search(obs, fft)
        log = ctx.last_worklog().splitlines()
    finally:
        ctx.set_worklog(False)

    assert cands and len(cands) == len(loop_cands)
    for a, b in zip(cands, loop_cands):
        assert (a[2], a[3], a[4], a[5]) == (b[2], b[3], b[4], b[5]), (a, b)
        assert _close(a[0], b[0], 1e-4) and _close(a[1], b[1], 1e-4), (a, b)
    assert len(log) == len(loop_log)
    for a, b in zip(log, loop_log):
        fa, fb = a.split(), b.split()
        assert fa[2:] == fb[2:], (a, b)
        assert _close(float(fa[0]), float(fb[0]), 1e-4) or abs(float(fa[0]) - float(fb[0])) <= 0.011
        assert abs(float(fa[1]) - float(fb[1])) <= 1e-3 * float(fb[1]) + 1.1e-4, (a, b)
    assert np.isfinite([c[0] for c in cands]).all()
