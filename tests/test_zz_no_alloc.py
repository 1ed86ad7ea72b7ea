"""ab_fderivs_vol_noalloc: plane generation that allocates no device memory.

It serves callers that cannot call cudaMalloc: pipelines that reserve all
device memory at start-up and forbid allocation in their processing loop,
hosts whose device memory belongs to another allocator, and stream-ordered
code in which an allocation would synchronise the device.  Its planes must
equal those of the allocating entry point ab_subharm_fderivs_vol within the
plane tolerance, on two calls in a row per bank (the second call reuses the
static scratch the first one left behind), for an acceleration search, a
jerk search (templates [nw][nz][L] with nw > 1) and the -locpow
normalisation.  A second pass over every call must leave the device's free
memory (cudaMemGetInfo) unchanged and give the same planes.  A template
buffer smaller than the bank is rejected with nothing written.

The static array's own limit (8192 work items, a 4096-point spectrum) is
above every bank the engine accepts, so its AB_ERR_BUDGET branch cannot be
reached with a valid search geometry and is not exercised here.

Collected last so that a failure here cannot hide the other tests."""
import ctypes as C

import numpy as np
import pytest

from presto_b200 import synth

pytestmark = pytest.mark.gpu
PTOL = 1e-4
DT = 64e-6
AB_ERR_ARG = -1

CASES = {
    "std": dict(N=1 << 17, seed=21, kw=dict(zmax=60, wmax=0, numharm=4),
                pulsars=[dict(r=1700.4, z=14.0, harms=[(0.08, 0.2)] * 3)], banks=[(1, 1), (4, 3)]),
    "jerk": dict(N=1 << 16, seed=22, kw=dict(zmax=20, wmax=40, numharm=2),
                 pulsars=[dict(r=900.2, z=6.0, w=25.0, harms=[(0.12, 0.0), (0.06, 0.5)])],
                 banks=[(1, 1), (2, 1)]),
    "locpow": dict(N=1 << 17, seed=23, kw=dict(zmax=60, wmax=0, numharm=4, locpow=True),
                   pulsars=[dict(r=1500.6, z=-9.0, harms=[(0.08, 0.2), (0.05, 0.9)])],
                   banks=[(1, 1), (2, 1)]),
}


def _prepare(ctx, ablib, torch):
    """Per case, bank and block: the allocating path's plane, the device
    templates and an output buffer filled with -1."""
    calls = []
    for name, c in CASES.items():
        fft = synth.spectrum(synth.time_series(c["N"], c["seed"], c["pulsars"]))
        obs = ablib.obs_init(ablib.make_params(c["N"], DT, fft.size, **c["kw"]))
        assert obs.norm_type == int(c["kw"].get("locpow", False))
        ctx.set_spectrum(obs, fft)
        dev_fft = torch.from_numpy(fft.view(np.float32).copy()).cuda()
        geo = {(g["numharm"], g["harmnum"]): g for g in ablib.bank_geometry(obs)}
        for (nh, hn) in c["banks"]:
            g = geo[(nh, hn)]
            tmpl = np.stack([np.stack([ctx.bank_kernel(obs, nh, hn, wi, zi)
                                       for zi in range(g["nz"])]) for wi in range(g["nw"])])
            assert tmpl.shape == (g["nw"], g["nz"], g["L"])
            dev_tmpl = torch.from_numpy(tmpl.view(np.float32).copy()).cuda()
            for k in (2, 9):                       # two calls in a row per bank
                lo = obs.rlo + k * obs.rstep
                meta, ref = ctx.subharm_fderivs_vol(obs, nh, hn, lo, lo + obs.rstep - 0.5)
                out = torch.full((ref.size,), -1.0, dtype=torch.float32, device="cuda")
                calls.append(dict(name=name, obs=obs, nh=nh, hn=hn, lo=lo, fft=dev_fft,
                                  tmpl=dev_tmpl, ntmpl_vals=tmpl.size, meta=meta, ref=ref,
                                  out=out))
    return calls


def _call(L, c, stream, tcap=None):
    m = __import__("presto_b200").accel.FFDotPows()
    rc = L.ab_fderivs_vol_noalloc(C.byref(c["obs"]), c["nh"], c["hn"], c["lo"],
                                  c["fft"].data_ptr(), c["tmpl"].data_ptr(),
                                  c["ntmpl_vals"] if tcap is None else tcap,
                                  c["out"].data_ptr(), c["out"].numel(),
                                  C.c_void_p(stream.cuda_stream), C.byref(m))
    return rc, m


def _check(c, m):
    meta = c["meta"]
    assert (m.rlo, m.zlo, m.wlo, m.numrs, m.numzs, m.numws) == (
        meta["rlo"], meta["zlo"], meta["wlo"], meta["numrs"], meta["numzs"], meta["numws"])
    ref = c["ref"]
    got = c["out"].cpu().numpy().reshape(ref.shape)
    ok = np.all(np.abs(got - ref) <= PTOL * (ref + max(float(ref.mean()), 1e-3)))
    assert ok, (c["name"], c["nh"], c["hn"], c["lo"])
    return got


def test_noalloc_matches_allocating_entry_point(ctx, ablib):
    import torch

    L = ablib.lib()
    stream = torch.cuda.current_stream()
    calls = _prepare(ctx, ablib, torch)
    first = []
    for c in calls:
        rc, m = _call(L, c, stream)
        assert rc == 0, (c["name"], rc)
        stream.synchronize()
        first.append(_check(c, m))
    # every call again: no device memory taken, the same planes
    for c in calls:
        c["out"].fill_(-1.0)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    metas = []
    for c in calls:
        rc, m = _call(L, c, stream)
        assert rc == 0, (c["name"], rc)
        metas.append(m)
    stream.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0, (free0, free1)
    for c, m, g in zip(calls, metas, first):
        assert np.array_equal(_check(c, m), g)


def test_noalloc_rejects_short_template_buffer(ctx, ablib):
    import torch

    L = ablib.lib()
    stream = torch.cuda.current_stream()
    c = _prepare(ctx, ablib, torch)[0]
    rc, _ = _call(L, c, stream, tcap=c["ntmpl_vals"] - 1)
    stream.synchronize()
    assert rc == AB_ERR_ARG
    assert bool(torch.all(c["out"] == -1.0))
