// ab_select.cuh -- exact order statistics of non-negative floats in shared
// memory (block medians of the search's normalisation and of de-reddening).
#pragma once
#include <cuda_runtime.h>

namespace ab {

// k-th smallest (0-based) of n non-negative floats in shared memory, exactly:
// a radix select over the IEEE bit patterns (which order like the values for
// x >= 0), four passes of 8-bit digits from the top.  Each pass histograms the
// digit of the candidates that match the prefix found so far (warp-aggregated
// shared atomics), and one warp scans the 256 counts for the digit holding
// rank k.  Called by every thread of the CTA (blockDim a multiple of 32).
__device__ __forceinline__ float select_rank(const float *a, int n, int k, unsigned *hist, unsigned *s_res)
{
    const int lane = threadIdx.x & 31;
    unsigned prefix = 0, mask = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0u;
        __syncthreads();
        for (int base = 0; base < n; base += blockDim.x) {
            const int i = base + threadIdx.x;
            unsigned key = 256u;                               // not a candidate
            if (i < n) {
                const unsigned u = __float_as_uint(a[i]);
                if ((u & mask) == prefix) key = (u >> shift) & 255u;
            }
            const unsigned peers = __match_any_sync(0xffffffffu, key);
            if (key < 256u && lane == __ffs(peers) - 1) atomicAdd(&hist[key], (unsigned) __popc(peers));
        }
        __syncthreads();
        if (threadIdx.x < 32) {
            // lane l owns digits 8l .. 8l+7
            unsigned c[8], tot = 0;
#pragma unroll
            for (int q = 0; q < 8; q++) {
                c[q] = hist[8 * lane + q];
                tot += c[q];
            }
            unsigned incl = tot;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            unsigned before = incl - tot;                     // candidates below this lane's digits
            const bool mine = (unsigned) k >= before && (unsigned) k < incl;
            if (mine) {
                unsigned acc = before;
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    if ((unsigned) k >= acc && (unsigned) k < acc + c[q]) {
                        s_res[0] = 8u * lane + q;
                        s_res[1] = (unsigned) k - acc;
                    }
                    acc += c[q];
                }
            }
        }
        __syncthreads();
        prefix |= s_res[0] << shift;
        mask |= 255u << shift;
        k = (int) s_res[1];
        __syncthreads();
    }
    return __uint_as_float(prefix);
}

}  // namespace ab
