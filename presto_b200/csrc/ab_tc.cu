// ab_tc.cu -- tensor-core (tcgen05) kernels.
//
// k_tc_gemm: one 128 x N tile of C = A . B^T with BF16 operands (optionally
// split into hi + lo parts, three products accumulated in FP32) staged in
// shared memory and accumulated in tensor memory: the self-test of the
// primitives.
//
// k_tc_pack / k_corr_tc: the segment correlation of subharm_fderivs_vol
// (src/accel_utils.c:1140-1193) evaluated as the banded template product it
// is, on the tensor cores.  With the data spread to even samples
// (spread_no_pad, src/corr_prep.c:62-74) and the template centred at index 0
// (place_complex_kernel, src/corr_prep.c:92-114), the power at plane column
// kk = 2a + p of template t is |y_p[a]|^2 with
//     y_p[a] = sum_c d[(a + p + c) mod numdata] * conj(resp_t[2 (hw_t - hw0 + c) + p]),
// c in [0, 2 hw0), d the normalised block data and resp_t the template's
// 4 hw_t response points (zero outside).  Per parity this is a real GEMM:
// M = output positions a, N = (re, im) rows of each template, K = taps with
// re/im interleaved.  Operands are split into 16-bit hi + lo parts -- BF16
// (8 significant bits each, FP32's exponent range) or FP16 (11 bits each, so
// about 2^-22 instead of 2^-16 relative, for operands below 65504 in
// magnitude) -- and the products hi.hi + hi.lo + lo.hi are accumulated in
// FP32 in tensor memory.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "ab_index.h"
#include "ab_kernels.h"
#include "ab_tc.cuh"

namespace ab {

__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16 &hi, __nv_bfloat16 &lo)
{
    hi = __float2bfloat16_rn(x);
    lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

// hi + lo 16-bit parts of x as raw bits: BF16 (F16 = false) or FP16
template <bool F16> __device__ __forceinline__ void split16(float x, uint16_t &hi, uint16_t &lo)
{
    if constexpr (F16) {
        const __half h = __float2half_rn(x);
        const __half l = __float2half_rn(x - __half2float(h));
        hi = __half_as_ushort(h);
        lo = __half_as_ushort(l);
    } else {
        __nv_bfloat16 h, l;
        split_bf16(x, h, l);
        hi = __bfloat16_as_ushort(h);
        lo = __bfloat16_as_ushort(l);
    }
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
    bool ok = tc::mbar_wait(&bar, 0, err, 2u);
    ok = __all_sync(0xffffffffu, ok);           // warp-uniform for the collective loads
    if (!ok) {
        // the output is discarded (the error word is set), but MMAs already
        // issued still read shared memory and write tensor memory: wait for
        // them (bounded again) before both are released
        tc::mbar_wait(&bar, 0, err, 16u);
    }
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

// ---------------------------------------------------------------------
// tensor-core correlation
// ---------------------------------------------------------------------

// Byte offset of element (row, k) in one K step (16 bf16 per row) of an
// operand in the no-swizzle K-major layout: 8-row groups of two 8 x 16 B core
// matrices (leading offset 128 B between the K halves, stride offset 256 B
// between row groups).
__device__ __forceinline__ uint32_t kstep_off(int row, int k)
{
    return (uint32_t) ((row >> 3) * 256 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// B operand of one bank's tiles.  CTA (x = parity * nks_max + s, y = tile)
// writes K step s: n rows (template q = row / 2; its re row, then its im
// row) x 16 bf16 (taps c_lo + 8 s + k / 2, re and im interleaved), hi part
// then lo part.  Rows re: (Re r, Im r); im: (-Im r, Re r) for the response
// point r, so that A . B^T gives Re and Im of d * conj(r).
template <bool F16>
__global__ void __launch_bounds__(256) k_tc_pack(const ab_bank b, const TcTile *tiles, int nks_max,
                                                 const int *perm, const float2 *raw, int stride,
                                                 unsigned char *pack)
{
    const TcTile tl = tiles[blockIdx.y];
    const int p = blockIdx.x / nks_max, s = blockIdx.x - p * nks_max;
    if (s >= tl.nks) return;
    unsigned char *dst = pack + tl.off + ((long long) p * tl.nks + s) * 64 * tl.n;
    for (int e = threadIdx.x; e < tl.n * 16; e += blockDim.x) {
        const int row = e >> 4, k = e & 15, q = row >> 1;
        float v = 0.f;
        if (q < tl.nt) {
            const int t = perm[tl.t0 + q];
            const int wi = t / b.nz, zi = t - wi * b.nz;
            const int hw = ab_resp_halfwidth((double) (-b.zmax + zi * AB_DZ),
                                             (double) (-b.wmax + wi * AB_DW));
            const int c = tl.c_lo + 8 * s + (k >> 1);
            const int idx = 2 * (hw - b.hw0 + c) + p;
            if (idx >= 0 && idx < 4 * hw) {
                const float2 r = raw[(long long) t * stride + idx];
                if ((row & 1) == 0) v = (k & 1) ? r.y : r.x;
                else v = (k & 1) ? r.x : -r.y;
            }
        }
        uint16_t h, l;
        split16<F16>(v, h, l);
        const uint32_t o = kstep_off(row, k);
        *reinterpret_cast<uint16_t *>(dst + o) = h;
        *reinterpret_cast<uint16_t *>(dst + 32 * tl.n + o) = l;
    }
}

cudaError_t launch_tc_pack(const ab_bank *b, const TcTile *tiles_dev, int ntiles, int nks_max,
                           const int *perm_dev, const float2 *raw, int stride,
                           unsigned char *pack, int fp16, cudaStream_t st)
{
    if (ntiles <= 0) return cudaSuccess;
    if (ntiles > 65535 || nks_max <= 0) return cudaErrorInvalidValue;
    dim3 grid(2 * nks_max, ntiles);
    if (fp16)
        k_tc_pack<true><<<grid, 256, 0, st>>>(*b, tiles_dev, nks_max, perm_dev, raw, stride, pack);
    else
        k_tc_pack<false><<<grid, 256, 0, st>>>(*b, tiles_dev, nks_max, perm_dev, raw, stride, pack);
    return cudaGetLastError();
}

size_t tc_corr_smem(int nks_max)
{
    // data rows (hi + lo) for the accumulators, then the template ring; at
    // least ~77 KB so that at most two CTAs (256 tensor-memory columns each)
    // share an SM: one's MMAs run while the other builds its data operand or
    // drains its accumulator
    size_t s = (size_t) (TC_ACC * TC_ATILE + 8 * nks_max) * 64 + (size_t) TC_STAGES * TC_CHUNK;
    return s < 77 * 1024 ? 77 * 1024 : s;
}

struct TcArgs {
    const ab_bank *banks;
    SearchConsts sc;
    BlockBatch bb;
    const TcItem *items;
    const TcTile *tiles;
    const int *perm;
    const float2 *dtime;
    long long dt_per_block;
    const unsigned char *pack;
    float *planes;
    long long plane_per_block;
    float *fullplane;
};

// One CTA = 128 threads: positions a0 .. a0 + 128 TC_ACC - 1 (accumulators of
// 128 rows, 256 tensor-memory columns each) of one parity, against one
// template tile.  Thread 0 streams the tile's K steps into a ring with bulk
// copies; thread 32 issues the MMAs (3 per accumulator and K step) and frees
// each stage with a commit; all four warps then read the accumulators back
// (warp w owns rows 32 w .. 32 w + 31) and store |y|^2.  The data operand is a
// Hankel matrix: row r holds d[a0 + p + c_lo + r + j], j < 8, so K step s of
// accumulator u is rows 8 s + 128 u .. + 127, one 8-row group (256 B) further
// per step.  Every wait is bounded and reports through sc.err.
template <bool F16>
__global__ void __launch_bounds__(128, 1) k_corr_tc(TcArgs a)
{
    extern __shared__ __align__(1024) unsigned char tsm[];
    __shared__ __align__(8) uint64_t full[TC_STAGES], empty[TC_STAGES], done;
    __shared__ uint32_t s_taddr;
    const TcItem it = a.items[blockIdx.x];
    const TcTile tl = a.tiles[it.tile];
    const ab_bank b = a.banks[tl.bank];
    const SearchConsts &sc = a.sc;
    const double startr = a.bb.startr[it.bi];
    const ab_hgeom g = ab_harm_geom(startr, startr + sc.rstep - AB_DR, b.numharm, b.harmnum,
                                    sc.obs_zlo, sc.obs_wlo, sc.corr_uselen);
    const int p = it.parity;
    long long lim = g.numrs;
    float *rowbase;
    long long rowstride;
    if (sc.inmem) {
        // full f-fdot plane (numws = 1), column 2 rlo + kk (fund_to_ffdotplane,
        // src/accel_utils.c:1219-1233); pre-pass blocks stop at clip_col
        rowbase = a.fullplane + g.rlo * AB_RDR;
        rowstride = sc.rlen;
        if (a.bb.is_pre) {
            long long room = sc.clip_col - g.rlo * AB_RDR;
            if (room < lim) lim = room;
        }
    } else {
        rowbase = a.planes + (long long) it.bi * a.plane_per_block + b.plane_off;
        rowstride = b.numrs_max;
        if (lim > b.numrs_max) lim = b.numrs_max;
    }
    const long long na_all = lim > p ? (lim - p + 1) / 2 : 0;
    const long long na_l = na_all - it.a0 < TC_ACC * TC_ATILE ? na_all - it.a0 : TC_ACC * TC_ATILE;
    if (na_l <= 0) return;                      // uniform over the CTA
    const int na = (int) na_l;
    const int nat = (na + TC_ATILE - 1) / TC_ATILE;
    const int nrows = TC_ATILE * nat + 8 * tl.nks;
    unsigned char *h_hi = tsm, *h_lo = tsm + (size_t) nrows * 32;
    unsigned char *ring = tsm + (size_t) nrows * 64;

    // data operand, hi and lo parts
    const int numdata = b.fftlen_ref / AB_NUMBETWEEN;
    const float2 *d = a.dtime + (long long) it.bi * a.dt_per_block + b.dtime_off;
    const int base = it.a0 + p + tl.c_lo;
    for (int e = threadIdx.x; e < nrows * 8; e += blockDim.x) {
        const int r = e >> 3, j = e & 7;
        const float2 v = __ldg(d + (base + r + j) % numdata);
        uint16_t hr, lr, hi_, li;
        split16<F16>(v.x, hr, lr);
        split16<F16>(v.y, hi_, li);
        const uint32_t o = kstep_off(r, 2 * j);
        *reinterpret_cast<uint32_t *>(h_hi + o) = (uint32_t) hr | ((uint32_t) hi_ << 16);
        *reinterpret_cast<uint32_t *>(h_lo + o) = (uint32_t) lr | ((uint32_t) li << 16);
    }
    if (threadIdx.x < 32) tc::tmem_alloc(&s_taddr, 256 * TC_ACC);
    if (threadIdx.x == 0) {
        for (int i = 0; i < TC_STAGES; i++) {
            tc::mbar_init(&full[i], 1);
            tc::mbar_init(&empty[i], 1);
        }
        tc::mbar_init(&done, 1);
    }
    tc::fence_smem_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t taddr = s_taddr;
    const uint32_t cbytes = 64u * (uint32_t) tl.n;
    const unsigned char *src = a.pack + tl.off + (long long) p * tl.nks * cbytes;

    if (threadIdx.x == 0) {
        // producer: template K steps into the ring
        int s = 0;
        for (; s < tl.nks; s++) {
            const int st = s % TC_STAGES;
            if (s >= TC_STAGES && !tc::mbar_wait(&empty[st], ((s / TC_STAGES) - 1) & 1, sc.err, 4u))
                break;
            tc::mbar_expect_tx(&full[st], cbytes);
            tc::bulk_g2s(ring + st * TC_CHUNK, src + (long long) s * cbytes, cbytes, &full[st]);
        }
        // copies in flight land before the CTA may exit
        for (int q = s > TC_STAGES ? s - TC_STAGES : 0; q < s; q++)
            tc::mbar_wait(&full[q % TC_STAGES], (q / TC_STAGES) & 1, sc.err, 4u);
    } else if (threadIdx.x == 32) {
        // MMA issuer
        const uint32_t idesc = F16 ? tc::idesc_f16_f32(TC_ATILE, tl.n) : tc::idesc_bf16_f32(TC_ATILE, tl.n);
        for (int s = 0; s < tl.nks; s++) {
            const int st = s % TC_STAGES;
            if (!tc::mbar_wait(&full[st], (s / TC_STAGES) & 1, sc.err, 4u)) break;
            tc::fence_after_sync();
            const unsigned char *bs = ring + st * TC_CHUNK;
            const uint64_t bh = tc::desc_k_nosw(bs, 128, 256);
            const uint64_t bl = tc::desc_k_nosw(bs + 32 * tl.n, 128, 256);
            for (int u = 0; u < nat; u++) {
                const uint64_t ah = tc::desc_k_nosw(h_hi + s * 256 + u * 4096, 128, 256);
                const uint64_t al = tc::desc_k_nosw(h_lo + s * 256 + u * 4096, 128, 256);
                const uint32_t dt = taddr + (uint32_t) (u * 256);
                tc::mma_bf16(dt, ah, bh, idesc, s > 0);
                tc::mma_bf16(dt, ah, bl, idesc, 1);
                tc::mma_bf16(dt, al, bh, idesc, 1);
            }
            tc::commit(&empty[st]);
        }
        tc::commit(&done);
    }
    __syncwarp();
    bool ok = tc::mbar_wait(&done, 0, sc.err, 8u);
    ok = __all_sync(0xffffffffu, ok);           // warp-uniform for the collective loads
    if (!ok) {
        // the batch's planes are discarded (the error word is set and the
        // search returns AB_ERR_CUDA), but MMAs already issued still read the
        // ring and the data operand and write tensor memory: wait for them
        // (bounded again) before shared and tensor memory are released
        tc::mbar_wait(&done, 0, sc.err, 16u);
    }
    tc::fence_after_sync();
    if (ok) {
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
        for (int u = 0; u < nat; u++) {
            const int al = u * TC_ATILE + 32 * w + lane;
            const bool valid = al < na;
            const long long kk = 2LL * (it.a0 + al) + p;
            for (int col = 0; col < tl.n; col += 8) {
                float v[8];
                tc::ld_x8(taddr + ((uint32_t) (32 * w) << 16) + (uint32_t) (u * 256 + col), v);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int tq = col / 2 + q;
                    if (valid && tq < tl.nt) {
                        const int t = a.perm[tl.t0 + tq];
                        rowbase[(long long) t * rowstride + kk] =
                            fmaf(v[2 * q], v[2 * q], v[2 * q + 1] * v[2 * q + 1]);
                    }
                }
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) tc::tmem_free(taddr, 256 * TC_ACC);
}

cudaError_t launch_corr_tc(const ab_bank *banks_dev, const SearchConsts &sc, const BlockBatch &bb,
                           const TcItem *items, int nitems, const TcTile *tiles, const int *perm,
                           const float2 *dtime, long long dt_per_block, const unsigned char *pack,
                           int nks_max, float *planes, long long plane_per_block, float *fullplane,
                           int fp16, cudaStream_t st)
{
    if (nitems <= 0) return cudaSuccess;
    const size_t smem = tc_corr_smem(nks_max);
    TcArgs a{banks_dev, sc, bb, items, tiles, perm, dtime, dt_per_block, pack, planes,
             plane_per_block, fullplane};
    // The attribute is the kernel's, shared by every host thread launching it
    // (a request pool's workers launch it with different sizes at once), so it
    // is set to one ceiling every launch fits under, never to this launch's
    // size: the 227 KB per block less the kernel's static shared memory.
    auto launch = [&](auto kern) -> cudaError_t {
        cudaFuncAttributes fa;
        cudaError_t e = cudaFuncGetAttributes(&fa, kern);
        if (e != cudaSuccess) return e;
        const size_t cap = 227 * 1024 - fa.sharedSizeBytes;
        if (smem > cap) return cudaErrorInvalidValue;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) cap);
        if (e != cudaSuccess) return e;
        kern<<<nitems, 128, smem, st>>>(a);
        return cudaGetLastError();
    };
    return fp16 ? launch(k_corr_tc<true>) : launch(k_corr_tc<false>);
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
