"""ab_fderivs_vol_noalloc: plane generation that allocates no device memory,
for callers that cannot call cudaMalloc (pre-reserved memory, a foreign
allocator, stream-ordered code).  Its planes must equal those of the
allocating entry point ab_subharm_fderivs_vol, on two calls in a row (the
second call reuses the static scratch the first one left behind).
Collected last so that a failure here cannot hide the other tests."""
import ctypes as C

import numpy as np
import pytest

from presto_b200 import synth

pytestmark = pytest.mark.gpu
PTOL = 1e-4


def test_noalloc_matches_allocating_entry_point(ctx, ablib):
    import torch

    N, dt = 1 << 17, 64e-6
    fft = synth.spectrum(synth.time_series(N, 21, [dict(r=1700.4, z=14.0, harms=[(0.08, 0.2)] * 3)]))
    obs = ablib.obs_init(ablib.make_params(N, dt, fft.size, zmax=60, wmax=0, numharm=4))
    ctx.set_spectrum(obs, fft)
    L = ablib.lib()
    dev_fft = torch.from_numpy(fft.view(np.float32).copy()).cuda()
    stream = torch.cuda.current_stream()
    geo = {(g["numharm"], g["harmnum"]): g for g in ablib.bank_geometry(obs)}
    starts = [obs.rlo + k * obs.rstep for k in (2, 9)]
    for (nh, hn) in [(1, 1), (4, 3)]:
        g = geo[(nh, hn)]
        tmpl = np.stack([np.stack([ctx.bank_kernel(obs, nh, hn, wi, zi) for zi in range(g["nz"])])
                         for wi in range(g["nw"])])
        dev_tmpl = torch.from_numpy(tmpl.view(np.float32).copy()).cuda()
        for lo in starts:                      # two calls in a row
            meta, ref = ctx.subharm_fderivs_vol(obs, nh, hn, lo, lo + obs.rstep - 0.5)
            out = torch.full((ref.size,), -1.0, dtype=torch.float32, device="cuda")
            m = ablib.accel.FFDotPows()
            rc = L.ab_fderivs_vol_noalloc(C.byref(obs), nh, hn, lo, dev_fft.data_ptr(),
                                          dev_tmpl.data_ptr(), out.data_ptr(), out.numel(),
                                          C.c_void_p(stream.cuda_stream), C.byref(m))
            assert rc == 0
            stream.synchronize()
            assert (m.rlo, m.zlo, m.wlo, m.numrs, m.numzs, m.numws) == (
                meta["rlo"], meta["zlo"], meta["wlo"], meta["numrs"], meta["numzs"], meta["numws"])
            got = out.cpu().numpy().reshape(ref.shape)
            assert np.all(np.abs(got - ref) <= PTOL * (ref + max(float(ref.mean()), 1e-3))), (nh, hn, lo)
