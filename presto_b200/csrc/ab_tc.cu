// ab_tc.cu -- tensor-core (tcgen05) kernels.
//
// k_tc_gemm: one 128 x N tile of C = A . B^T with BF16 operands (optionally
// split into hi + lo parts, three products accumulated in FP32) staged in
// shared memory and accumulated in tensor memory.  It is the building block of
// the split-precision correlation and its self-test.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "ab_tc.cuh"

namespace ab {

__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16 &hi, __nv_bfloat16 &lo)
{
    hi = __float2bfloat16_rn(x);
    lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

// 128 threads.  A: [128][K], B: [N][K] row-major FP32 in global memory,
// C: [128][N].  K % 16 == 0, K <= 256, N % 16 == 0, 16 <= N <= 256.
__global__ void __launch_bounds__(128) k_tc_gemm(const float *A, const float *B, float *C, int N, int K,
                                                 int split, unsigned *err)
{
    extern __shared__ __align__(128) unsigned char tsm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t s_taddr;
    const int nA = 128 * K * 2, nB = N * K * 2;      // bytes of one bf16 tile
    unsigned char *a_hi = tsm, *a_lo = tsm + nA, *b_hi = tsm + 2 * nA, *b_lo = tsm + 2 * nA + nB;
    for (int e = threadIdx.x; e < 128 * K; e += blockDim.x) {
        int r = e / K, k = e - r * K;
        __nv_bfloat16 h, l;
        split_bf16(A[e], h, l);
        uint32_t o = tc::kmajor_off(r, k, K);
        *reinterpret_cast<__nv_bfloat16 *>(a_hi + o) = h;
        *reinterpret_cast<__nv_bfloat16 *>(a_lo + o) = l;
    }
    for (int e = threadIdx.x; e < N * K; e += blockDim.x) {
        int r = e / K, k = e - r * K;
        __nv_bfloat16 h, l;
        split_bf16(B[e], h, l);
        uint32_t o = tc::kmajor_off(r, k, K);
        *reinterpret_cast<__nv_bfloat16 *>(b_hi + o) = h;
        *reinterpret_cast<__nv_bfloat16 *>(b_lo + o) = l;
    }
    uint32_t ncols = 32;
    while ((int) ncols < N) ncols <<= 1;
    if (threadIdx.x < 32) tc::tmem_alloc(&s_taddr, ncols);
    if (threadIdx.x == 0) tc::mbar_init(&bar, 1);
    tc::fence_smem_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t taddr = s_taddr;
    if (threadIdx.x == 0) {
        const uint32_t idesc = tc::idesc_bf16_f32(128, N);
        const uint32_t sboA = (K / 8) * 128, sboB = (K / 8) * 128;
        for (int ks = 0; ks < K / 16; ks++) {
            uint64_t ah = tc::desc_k_nosw(a_hi + ks * 256, 128, sboA);
            uint64_t bh = tc::desc_k_nosw(b_hi + ks * 256, 128, sboB);
            tc::mma_bf16(taddr, ah, bh, idesc, ks > 0);
            if (split) {
                uint64_t al = tc::desc_k_nosw(a_lo + ks * 256, 128, sboA);
                uint64_t bl = tc::desc_k_nosw(b_lo + ks * 256, 128, sboB);
                tc::mma_bf16(taddr, ah, bl, idesc, 1);
                tc::mma_bf16(taddr, al, bh, idesc, 1);
            }
        }
        tc::commit(&bar);
    }
    const bool ok = tc::mbar_wait(&bar, 0, err, 2u);
    tc::fence_after_sync();
    if (ok) {
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int row = 32 * w + lane;
        for (int c = 0; c < N; c += 8) {
            float v[8];
            tc::ld_x8(taddr + ((uint32_t) (32 * w) << 16) + (uint32_t) c, v);
#pragma unroll
            for (int i = 0; i < 8; i++) C[row * N + c + i] = v[i];
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) tc::tmem_free(taddr, ncols);
}

cudaError_t launch_tc_gemm(const float *A, const float *B, float *C, int N, int K, int split,
                           unsigned *err, cudaStream_t st)
{
    if (K % 16 || K < 16 || K > 256 || N % 16 || N < 16 || N > 256) return cudaErrorInvalidValue;
    size_t smem = (size_t) 2 * (128 + N) * K * 2;
    cudaFuncSetAttribute(k_tc_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    k_tc_gemm<<<1, 128, smem, st>>>(A, B, C, N, K, split, err);
    return cudaGetLastError();
}

}  // namespace ab
