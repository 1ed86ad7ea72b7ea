"""tcgen05 building block of the split-precision correlation: a 128 x N tile
of A . B^T from BF16 operands with FP32 accumulation in tensor memory."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bf16(x):
    """Round float32 to bfloat16 (round to nearest even), back to float64."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


@pytest.mark.parametrize("N,K", [(128, 64), (64, 128), (256, 32)])
def test_tc_gemm(ctx, ablib, N, K):
    rng = np.random.default_rng(N + K)
    A = rng.standard_normal((128, K)).astype(np.float32)
    B = rng.standard_normal((N, K)).astype(np.float32)
    L = ablib.lib()
    out = {}
    for split in (0, 1):
        Cm = np.zeros((128, N), np.float32)
        rc = L.ab_tc_gemm(ctx.ptr, A.ctypes.data, B.ctypes.data, Cm.ctypes.data, N, K, split)
        assert rc == 0, L.ab_ctx_last_error(ctx.ptr)
        out[split] = Cm.astype(np.float64)
    exact = A.astype(np.float64) @ B.astype(np.float64).T
    single = _bf16(A) @ _bf16(B).T
    scale = np.sqrt(K)
    assert np.max(np.abs(out[0] - single)) < 1e-4 * scale
    # split: each product keeps ~16 mantissa bits (the lo.lo term and the
    # rounding of the lo parts are dropped): ~2^-15 per product, summed over K
    assert np.max(np.abs(out[1] - exact)) < 2 ** -14 * scale * 4
    assert np.max(np.abs(out[0] - exact)) > 20 * np.max(np.abs(out[1] - exact))
