// ab_dedisp.cu -- subband dedispersion on the device: the DM-trial producer
// of accelsearch's input (prepsubband, src/prepsubband.c:365-450 with
// src/dispersion.c:165-232 and the downsampling of :985-1003).
//
// Two stages, as prepsubband forms them, each output element summed in the
// reference's order so that the results are its bits:
//   subbands  S[s][t] = sum_{c in subband s, ascending} X[t + cd[c]][c]
//             (dedisp_subbands), then the downsampling
//             D[s][u] = 0 + (sum_{k < ds} S[s][u ds + k]) / ds;
//   DMs       out[d][u] = -0 + sum_{s ascending} D[s][u + off[d][s]]
//             (float_dedisp with approx_mean 0),
// samples past the end of the data reading zero (the reference's zeroed
// final block).  The input spectra X are time-major (all channels of a
// sample together, channels ascending in frequency) and are read once, in
// row segments of a subband's channels.  The DM stage gives each thread 4 or
// 8 output samples of 32, 16 or 8 consecutive DMs, which read nearby samples
// of the same subband: one shared-memory window per subband serves them all.
#include <cuda_runtime.h>
#include <stdint.h>

#include "ab_kernels.h"

namespace ab {
namespace {

constexpr int SB_TILE = 256;            // downsampled samples per subband CTA
constexpr int DM_THREADS = 128;         // threads per DM CTA
constexpr int STAGES = 4;               // subband windows in flight per DM CTA

// D[s][u] for u in [u0, u0 + SB_TILE) of subband s, from the time-major
// spectra x[t][c]: the rows the tile reads (its samples plus the subband's
// largest channel delay) of the subband's channels are staged in shared
// memory (each row's channels contiguous in memory, the shared rows padded to
// an odd stride so that consecutive samples hit different banks), then each
// thread sums its sample's channels and its ds samples in the reference's
// order.  blockIdx.x = sample tile * nsub + subband: the subbands of one tile
// run together, so each spectra row is fetched from memory once.
//
// CPS > 0: CPS channels per subband known at compile time (a multiple of 4,
// nchan too, x 16-byte aligned): each thread loads one fixed 16-byte column
// of every (SB_TILE / (CPS / 4))-th row, two loads in flight, and keeps its
// channels' delays in registers.  CPS == 0: any cps, one float per load.
template <int CPS>
__global__ void __launch_bounds__(SB_TILE) k_dd_subbands(const float *x, long long nspec, int nchan,
                                                         const int *cd, int cps, int ds,
                                                         long long nout, int maxcd, float *D)
{
    extern __shared__ float rows[];                    // [nrows][pitch]
    const int nsub = nchan / cps;
    const int s = (int) (blockIdx.x % (unsigned) nsub);
    const long long u0 = (long long) (blockIdx.x / (unsigned) nsub) * SB_TILE;
    const long long t_lo = u0 * ds;
    const int nrows = SB_TILE * ds + maxcd;
    if constexpr (CPS > 0) {
        constexpr int Q = CPS / 4, R = SB_TILE / Q, P = CPS | 1, UNR = 2;
        static_assert(CPS % 4 == 0 && SB_TILE % Q == 0, "16-byte columns tile the rows");
        const float4 *src4 = reinterpret_cast<const float4 *>(x + (long long) s * CPS) + threadIdx.x % Q;
        const long long rs4 = nchan >> 2;
        float *dst = rows + 4 * (threadIdx.x % Q);
        for (int r = threadIdx.x / Q; r < nrows; r += UNR * R) {
            float4 v[UNR];
#pragma unroll
            for (int k = 0; k < UNR; k++) {
                const int rr = r + k * R;
                const long long t = t_lo + rr;
                v[k] = rr < nrows && t < nspec ? __ldg(src4 + t * rs4)
                                               : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
#pragma unroll
            for (int k = 0; k < UNR; k++) {
                const int rr = r + k * R;
                if (rr < nrows) {
                    float *d = dst + rr * P;
                    d[0] = v[k].x;
                    d[1] = v[k].y;
                    d[2] = v[k].z;
                    d[3] = v[k].w;
                }
            }
        }
        int c[CPS];                                    // shared offset of channel j's delayed row
#pragma unroll
        for (int j = 0; j < CPS; j++) c[j] = __ldg(cd + s * CPS + j) * P + j;
        __syncthreads();
        const long long u = u0 + threadIdx.x;
        if (u >= nout) return;
        float ftmp = 0.0f;
        for (int k = 0; k < ds; k++) {
            const float *rp = rows + (threadIdx.x * ds + k) * P;
            float acc = 0.0f;
#pragma unroll
            for (int j = 0; j < CPS; j++) acc = __fadd_rn(acc, rp[c[j]]);
            ftmp = __fadd_rn(ftmp, acc);
        }
        D[(long long) s * nout + u] = ds == 1 ? ftmp : __fadd_rn(0.0f, __fdiv_rn(ftmp, (float) ds));
    } else {
        __shared__ int s_cd[1024];
        const int pitch = cps | 1;
        for (int j = threadIdx.x; j < cps; j += blockDim.x) s_cd[j] = cd[s * cps + j];
        const float *src = x + (long long) s * cps;
        for (int e = threadIdx.x; e < nrows * cps; e += blockDim.x) {
            const int r = e / cps, j = e - r * cps;
            const long long t = t_lo + r;
            rows[r * pitch + j] = t < nspec ? __ldg(src + t * nchan + j) : 0.0f;
        }
        __syncthreads();
        const long long u = u0 + threadIdx.x;
        if (u >= nout) return;
        float ftmp = 0.0f;
        for (int k = 0; k < ds; k++) {
            const int r = threadIdx.x * ds + k;
            float acc = 0.0f;
            for (int j = 0; j < cps; j++) acc = __fadd_rn(acc, rows[(r + s_cd[j]) * pitch + j]);
            ftmp = __fadd_rn(ftmp, acc);
        }
        D[(long long) s * nout + u] = ds == 1 ? ftmp : __fadd_rn(0.0f, __fdiv_rn(ftmp, (float) ds));
    }
}

// 4-byte asynchronous copy global -> shared; src_bytes 0 writes a zero
__device__ __forceinline__ void cp_async4(float *dst, const float *src, int src_bytes)
{
    const unsigned d = (unsigned) __cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src),
                 "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// out[d][u] for G consecutive DMs and the SPT * DM_THREADS samples of one
// tile; thread i adds samples i, i + DM_THREADS, ... (so that a warp's reads of
// a window are consecutive words).  blockIdx.x = sample tile * ngroups + DM
// group: the DM groups of one tile run together and share its subband rows in
// L2.  Per subband, the window of D the group reads (the tile's samples plus
// the spread of the group's offsets, zero past the end of the data) is copied
// into a ring of STAGES shared-memory windows by asynchronous copies issued
// STAGES - 1 subbands ahead, so that the copies of later subbands are in
// flight while the threads add the current one.
template <int G, int SPT>
__global__ void __launch_bounds__(DM_THREADS) k_dd_dms(const float *D, long long nout, int nsub,
                                                       const int *off, int ndm, int ngroups,
                                                       int wcap, float *out)
{
    constexpr int TILE = DM_THREADS * SPT;
    extern __shared__ __align__(16) int dsm[];
    int *s_rel = dsm;                                  // [nsub][G] offset - window start
    int *s_lo = s_rel + nsub * G;                      // [nsub] window start
    int *s_len = s_lo + nsub;                          // [nsub] window length (<= wcap)
    float *win = reinterpret_cast<float *>(s_len + nsub);   // [STAGES][wcap]
    const int grp = (int) (blockIdx.x % (unsigned) ngroups);
    const long long u0 = (long long) (blockIdx.x / (unsigned) ngroups) * TILE;
    const int d0 = grp * G;
    const int nd = min(G, ndm - d0);
    for (int s = threadIdx.x; s < nsub; s += blockDim.x) {
        int lo = off[(long long) d0 * nsub + s], hi = lo;
        for (int d = 1; d < nd; d++) {
            const int o = off[(long long) (d0 + d) * nsub + s];
            lo = min(lo, o);
            hi = max(hi, o);
        }
        s_lo[s] = lo;
        s_len[s] = TILE + hi - lo;
        for (int d = 0; d < G; d++)
            s_rel[s * G + d] = d < nd ? off[(long long) (d0 + d) * nsub + s] - lo : 0;
    }
    __syncthreads();
    auto issue = [&](int s) {
        if (s < nsub) {
            float *w = win + (s % STAGES) * wcap;
            const long long base = u0 + s_lo[s];
            const float *row = D + (long long) s * nout + base;
            const long long room = nout - base;
            const int len = s_len[s];
            for (int i = threadIdx.x; i < len; i += DM_THREADS) {
                const bool in = i < room;
                cp_async4(w + i, in ? row + i : D, in ? 4 : 0);
            }
        }
        cp_async_commit();                             // empty groups keep the count uniform
    };
#pragma unroll
    for (int p = 0; p < STAGES - 1; p++) issue(p);
    float acc[SPT][G];
#pragma unroll
    for (int k = 0; k < SPT; k++)
#pragma unroll
        for (int d = 0; d < G; d++) acc[k][d] = -0.0f;
    for (int s = 0; s < nsub; s++) {
        cp_async_wait<STAGES - 2>();                   // subband s's window has landed
        __syncthreads();                               // ... for every thread; stage s-1 is free
        issue(s + STAGES - 1);
        const float *w = win + (s % STAGES) * wcap + threadIdx.x;
        const int4 *rel = reinterpret_cast<const int4 *>(s_rel + s * G);
#pragma unroll
        for (int q = 0; q < G / 4; q++) {
            const int4 r = rel[q];
#pragma unroll
            for (int k = 0; k < SPT; k++) {
                acc[k][4 * q + 0] = __fadd_rn(acc[k][4 * q + 0], w[k * DM_THREADS + r.x]);
                acc[k][4 * q + 1] = __fadd_rn(acc[k][4 * q + 1], w[k * DM_THREADS + r.y]);
                acc[k][4 * q + 2] = __fadd_rn(acc[k][4 * q + 2], w[k * DM_THREADS + r.z]);
                acc[k][4 * q + 3] = __fadd_rn(acc[k][4 * q + 3], w[k * DM_THREADS + r.w]);
            }
        }
    }
    cp_async_wait<0>();
#pragma unroll
    for (int k = 0; k < SPT; k++) {
        const long long u = u0 + threadIdx.x + k * DM_THREADS;
        if (u >= nout) continue;
#pragma unroll
        for (int d = 0; d < G; d++)
            if (d < nd) out[(long long) (d0 + d) * nout + u] = acc[k][d];
    }
}

// largest spread of one subband's offsets over a group of g consecutive DMs
int group_spread(const int *off, int ndm, int nsub, int g)
{
    int m = 0;
    for (int d0 = 0; d0 < ndm; d0 += g)
        for (int s = 0; s < nsub; s++) {
            int lo = off[(size_t) d0 * nsub + s], hi = lo;
            for (int d = d0 + 1; d < ndm && d < d0 + g; d++) {
                lo = off[(size_t) d * nsub + s] < lo ? off[(size_t) d * nsub + s] : lo;
                hi = off[(size_t) d * nsub + s] > hi ? off[(size_t) d * nsub + s] : hi;
            }
            m = hi - lo > m ? hi - lo : m;
        }
    return m;
}

size_t dms_smem(int g, int nsub, int wcap)
{
    return sizeof(int) * ((size_t) nsub * g + 2 * (size_t) nsub) + sizeof(float) * STAGES * (size_t) wcap;
}

// DMs per thread G and samples per thread SPT, as measured best on B200 for
// 1024 channels x 2^20 spectra x 128 DMs: 32 x 4, 16 x 4, 8 x 8
constexpr int dm_spt(int g) { return g == 8 ? 8 : 4; }
constexpr int dm_tile(int g) { return DM_THREADS * dm_spt(g); }

template <int G>
cudaError_t launch_dms(const float *D, long long nout, int nsub, const int *off, int ndm, int wcap,
                       size_t smem, float *out, cudaStream_t st)
{
    constexpr int SPT = dm_spt(G);
    const int ngroups = (ndm + G - 1) / G;
    const long long ntiles = (nout + dm_tile(G) - 1) / dm_tile(G);
    if (ntiles * ngroups > 0x7FFFFFFFLL) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(k_dd_dms<G, SPT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess) return e;
    k_dd_dms<G, SPT><<<(unsigned) (ntiles * ngroups), DM_THREADS, smem, st>>>(D, nout, nsub, off,
                                                                              ndm, ngroups, wcap, out);
    return cudaGetLastError();
}

template <int CPS>
cudaError_t launch_sub(const float *x, long long nspec, int nchan, const int *cd, int cps, int ds,
                       long long nout, int maxcd, float *D, size_t smem, unsigned grid,
                       cudaStream_t st)
{
    cudaError_t e = cudaFuncSetAttribute(k_dd_subbands<CPS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess) return e;
    k_dd_subbands<CPS><<<grid, SB_TILE, smem, st>>>(x, nspec, nchan, cd, cps, ds, nout, maxcd, D);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_dedisp(const float *x, long long nspec, int nchan, const int *cd, int maxcd,
                          int nsub, int ds, const int *off, const int *off_host, int ndm, float *D,
                          float *out, cudaStream_t st)
{
    if (nspec < 1 || nchan < 1 || nsub < 1 || nchan % nsub || ds < 1 || ndm < 1 || maxcd < 0 ||
        nsub > 1024)
        return cudaErrorInvalidValue;
    const int cps = nchan / nsub;
    const long long nout = nspec / ds;
    const size_t smem = sizeof(float) * (size_t) (SB_TILE * ds + maxcd) * (size_t) (cps | 1);
    const long long stiles = (nout + SB_TILE - 1) / SB_TILE;
    if (nout < 1 || cps > 1024 || stiles * nsub > 0x7FFFFFFFLL || smem > 200 * 1024)
        return cudaErrorInvalidValue;
    // DMs per thread: the most of 32 / 16 / 8 (no more than the trials, in
    // steps of 8) whose windows leave room for four CTAs per SM; else the
    // fewest that fit at all
    int g = 0;
    size_t smem2 = 0;
    const int gs[3] = {32, 16, 8};
    for (int i = 0; i < 3 && !g; i++) {
        if (gs[i] > 8 && gs[i] >= ndm + 8) continue;
        const size_t m = dms_smem(gs[i], nsub, dm_tile(gs[i]) + group_spread(off_host, ndm, nsub, gs[i]));
        if (m <= 48 * 1024) g = gs[i], smem2 = m;
    }
    if (!g) {
        g = 8;
        smem2 = dms_smem(8, nsub, dm_tile(8) + group_spread(off_host, ndm, nsub, 8));
        if (smem2 > 200 * 1024) return cudaErrorInvalidValue;
    }
    const int wcap = dm_tile(g) + group_spread(off_host, ndm, nsub, g);
    const bool vec = nchan % 4 == 0 && ((uintptr_t) x & 15) == 0;
    const unsigned grid = (unsigned) (stiles * nsub);
    cudaError_t e;
    switch (vec ? cps : 0) {
    case 4: e = launch_sub<4>(x, nspec, nchan, cd, cps, ds, nout, maxcd, D, smem, grid, st); break;
    case 8: e = launch_sub<8>(x, nspec, nchan, cd, cps, ds, nout, maxcd, D, smem, grid, st); break;
    case 16: e = launch_sub<16>(x, nspec, nchan, cd, cps, ds, nout, maxcd, D, smem, grid, st); break;
    case 32: e = launch_sub<32>(x, nspec, nchan, cd, cps, ds, nout, maxcd, D, smem, grid, st); break;
    default: e = launch_sub<0>(x, nspec, nchan, cd, cps, ds, nout, maxcd, D, smem, grid, st); break;
    }
    if (e != cudaSuccess) return e;
    switch (g) {
    case 32: return launch_dms<32>(D, nout, nsub, off, ndm, wcap, smem2, out, st);
    case 16: return launch_dms<16>(D, nout, nsub, off, ndm, wcap, smem2, out, st);
    default: return launch_dms<8>(D, nout, nsub, off, ndm, wcap, smem2, out, st);
    }
}

}  // namespace ab
