"""Edge cases through the C ABI: a search with nothing above threshold, an
empty candidate list to polish, the full pipeline on pure noise, and the
shortest spectrum the geometry allows."""
import numpy as np
import pytest

from presto_b200 import synth

pytestmark = pytest.mark.gpu
DT = 64e-6


def test_noise_search_at_high_sigma_is_empty(ctx, ablib):
    N = 1 << 18
    ft = synth.spectrum(synth.time_series(N, 99))
    obs = ablib.obs_init(ablib.make_params(N, DT, ft.size, zmax=20, numharm=4, sigma=30.0))
    assert ctx.search(obs, ft) == []
    assert ctx.optimize_cands(obs, ft, []) == []
    res = ablib.AccelSearch(zmax=20, numharm=4, sigma=30.0, ctx=ctx).run(ft, N, DT)
    assert (res["cands"], res["polished"], res["props"]) == ([], [], [])


@pytest.mark.parametrize("inmem", [False, True])
def test_short_spectrum(ctx, ablib, oracle, inmem):
    """A spectrum of a few blocks: the device and the oracle agree."""
    import os
    N = 1 << 13
    ft = synth.spectrum(synth.time_series(N, 7, [dict(r=700.3, z=3.0, harms=[(0.3, 0.0)])]))
    kw = dict(zmax=10, numharm=2, wmax=None if inmem else 0)
    obs = ablib.obs_init(ablib.make_params(N, DT, ft.size, **kw))
    assert obs.inmem == int(inmem)
    dev = ctx.search(obs, ft)
    orc, _, _ = oracle.accelsearch(oracle.make_params(N, DT, ft.size, **kw), ft,
                                   nthreads=os.cpu_count() or 1)
    assert len(dev) == len(orc) and len(dev) > 0
    for d, o in zip(dev, orc):
        assert d[2] == o[2] and abs(d[3] - o[3]) < 1e-3 and abs(d[4] - o[4]) < 1e-3
        assert abs(d[0] - o[0]) <= 1e-4 * o[0]
