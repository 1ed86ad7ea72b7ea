"""Batched / served searches (ab_pool): every request's candidate list is the
same when searched alone on a plain context and when searched in a mix of
concurrent requests of different lengths, zmax, wmax and numharm."""
import numpy as np
import pytest

from presto_b200 import serve, synth

pytestmark = pytest.mark.gpu
DT = 64e-6

MIX = [
    dict(N=1 << 17, zmax=60, numharm=8, pulsars=[dict(r=2500.3, z=10.0, harms=[(0.06, 0.2)] * 4)]),
    dict(N=1 << 16, zmax=20, numharm=2, pulsars=[dict(r=700.6, z=-4.0, harms=[(0.1, 0.0)] * 2)]),
    dict(N=(1 << 17) + 2046, zmax=100, numharm=4, wmax=0, pulsars=[]),
    dict(N=1 << 16, zmax=20, numharm=2, wmax=40,
         pulsars=[dict(r=900.2, z=6.0, w=25.0, harms=[(0.12, 0.0), (0.06, 0.5)])]),
    dict(N=1 << 17, zmax=0, numharm=4, pulsars=[dict(r=3001.0, z=0.0, harms=[(0.05, 0.0)] * 3)]),
    dict(N=1 << 18, zmax=60, numharm=16, wmax=0,
         pulsars=[dict(r=9000.4, z=30.0, harms=[(0.03, 0.1)] * 8)]),
]


def _case(i, c):
    fft = synth.spectrum(synth.time_series(c["N"], 300 + i, c["pulsars"]))
    opts = dict(zmax=c["zmax"], numharm=c["numharm"])
    if "wmax" in c:
        opts["wmax"] = c["wmax"]
    return fft, opts


def test_pool_results_equal_alone(ctx, ablib):
    cases = [_case(i, c) for i, c in enumerate(MIX)]
    alone = []
    for (fft, opts), c in zip(cases, MIX):
        obs = ablib.obs_init(ablib.make_params(c["N"], DT, fft.size, **opts))
        alone.append(ctx.search(obs, fft))
    pool = serve.SearchPool(0, nworkers=3)
    try:
        # two rounds, submitted all at once so that requests overlap
        tickets = [pool.submit(fft, c["N"], DT, **opts) for (fft, opts), c in zip(cases * 2, MIX * 2)]
        got = [pool.wait(t) for t in tickets]
        st = pool.stats()
    finally:
        pool.close()
    assert st["completed"] == len(tickets)
    assert st["p99_ms"] >= st["p50_ms"] > 0
    for k, (cands, lat) in enumerate(got):
        assert cands == alone[k % len(MIX)], k
        assert lat > 0
    assert sum(len(a) for a in alone) > 0


@pytest.mark.parametrize("path", ["bf16", "fp16"])
def test_pool_tensor_core_mix_equal_alone(ablib, path):
    """The same mix on the tensor-core correlation: workers launch the
    contraction concurrently with different operand widths (different
    dynamic shared-memory sizes), and every result equals the request alone
    on a plain context of the same path."""
    code = ablib.CORR_TC_SPLIT_BF16 if path == "bf16" else ablib.CORR_TC_SPLIT_FP16
    cases = [_case(i, c) for i, c in enumerate(MIX)]
    plain = ablib.Context(0)
    try:
        plain.set_corr_path(code)
        alone = [plain.search(ablib.obs_init(ablib.make_params(c["N"], DT, fft.size, **opts)), fft)
                 for (fft, opts), c in zip(cases, MIX)]
    finally:
        plain.close()
    pool = serve.SearchPool(0, nworkers=3)
    try:
        pool.set_corr_path(code)
        tickets = [pool.submit(fft, c["N"], DT, **opts) for (fft, opts), c in zip(cases * 3, MIX * 3)]
        got = [pool.wait(t)[0] for t in tickets]
    finally:
        pool.close()
    for k, cands in enumerate(got):
        assert cands == alone[k % len(MIX)], k


def test_pool_rejects_oversized_request(ablib):
    pool = serve.SearchPool(0, nworkers=1, hbm_budget=12 << 30)
    try:
        fft = np.zeros(1 << 22, np.complex64)
        with pytest.raises(ablib.AccelError):
            pool.submit(fft, 1 << 23, DT, zmax=600, inmem=True)
    finally:
        pool.close()
