// ab_norm.cuh -- spectrum normalisation helpers shared by the search's block
// preparation and the time-series path.
#pragma once
#include <cuda_runtime.h>

namespace ab {

// invsqrtf (src/misc_utils.c:291-302): the published fast inverse square
// root, one Newton step, in float with explicit rounding.
__device__ __forceinline__ float fast_invsqrtf(float x)
{
    const float y = __int_as_float(0x5f3759df - (__float_as_int(x) >> 1));
    const float t = __fmul_rn(__fmul_rn(__fmul_rn(0.5f, x), y), y);
    return __fmul_rn(y, __fsub_rn(1.5f, t));
}

// -locpow: the factor invsqrtf(local power) that scales bin i of a block's
// window of numdata powers pw (src/accel_utils.c:1100-1113).  corr_loc_pow
// (src/corr_routines.c:309-366) correlates the powers with a double top-hat
// of 20 taps at offsets +-6..+-15 bins, each (numdata / 2) / NUMLOCPOWAVG in
// integer arithmetic, through real FFTs whose round trip carries 2 / numdata:
//   local[i] = (2 / numdata) floor(numdata / 40) sum_{6 <= |j| <= 15} pw[i + j],
// and the first and last 15 bins take the value of the nearest bin 15 from
// the edge.  The sum is formed exactly here (the reference's FP32 FFTs round
// it); no tap wraps, since every bin used lies 15 or more from the edges.
__device__ __forceinline__ float locpow_invsqrt(const float *pw, int numdata, int i)
{
    constexpr int khw = 20 / 2 + 5;                    // NUMLOCPOWAVG / 2 + DELTAAVGBINS
    const int c = i < khw ? khw : (i > numdata - 1 - khw ? numdata - 1 - khw : i);
    double s = 0.0;
#pragma unroll
    for (int j = 6; j <= khw; j++) s += (double) pw[c - j] + (double) pw[c + j];
    const double normal = (double) ((numdata / 2) / 20);
    const float local = (float) (s * normal * (2.0 / (double) numdata));
    return fast_invsqrtf(local);
}

}  // namespace ab
