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
// 128-byte row segments of 32 channels.  The DM stage gives each thread 8
// output samples of 16 or 8 consecutive DMs, which read nearby samples of
// the same subband: one shared-memory window per subband serves them all.
// D's rows are padded to a multiple of 4 floats (dedisp_sub_pitch) so that
// the windows move in 16-byte copies.
#include <cuda_runtime.h>
#include <stdint.h>

#include "ab_kernels.h"

namespace ab {

long long dedisp_sub_pitch(long long nout) { return (nout + 3) & ~3LL; }

namespace {

constexpr int SB_TILE = 256;            // downsampled samples per subband CTA
constexpr int STAGES = 4;               // subband windows in flight per DM CTA
constexpr int DM_THREADS = 64;          // threads per DM CTA
constexpr int DM_SPT = 8;               // samples per DM thread
constexpr int DM_TILE = DM_THREADS * DM_SPT;

// D[s][u] for u in [u0, u0 + SB_TILE) of the CW / CPS subbands of channels
// [c0, c0 + CW), from the time-major spectra x[t][c].  The rows the tile reads
// (its samples plus the largest channel delay) of those channels are staged in
// shared memory, CW + 1 words apart: each thread loads one fixed 16-byte
// column of every (SB_TILE / (CW / 4))-th row, three loads in flight, and with
// CW = 32 a warp's stores and the sums' reads both land in 32 distinct banks.
// Each thread then sums its sample's channels of each subband and its ds
// samples in the reference's order.  blockIdx.x = sample tile * (nchan / CW)
// + channel group: the groups of one tile run together, so each spectra row is
// fetched from memory once.  Requires nchan % CW == 0 and x 16-byte aligned.
template <int CW, int CPS>
__global__ void __launch_bounds__(SB_TILE) k_dd_subbands(const float *x, long long nspec, int nchan,
                                                         const int *cd, int ds, long long nout,
                                                         long long pitch, int maxcd, float *D)
{
    constexpr int GS = CW / CPS, Q = CW / 4, R = SB_TILE / Q, P = CW + 1, UNR = 3;
    static_assert(CW % 4 == 0 && CW % CPS == 0 && SB_TILE % Q == 0, "16-byte columns tile the rows");
    extern __shared__ float rows[];                    // [nrows][P]
    const int ngrp = nchan / CW;
    const int grp = (int) (blockIdx.x % (unsigned) ngrp);
    const long long u0 = (long long) (blockIdx.x / (unsigned) ngrp) * SB_TILE;
    const long long t_lo = u0 * ds;
    const int nrows = SB_TILE * ds + maxcd;
    const float4 *src4 = reinterpret_cast<const float4 *>(x + (long long) grp * CW) + threadIdx.x % Q;
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
    int c[CW];                                         // shared offset of channel j's delayed row
#pragma unroll
    for (int j = 0; j < CW; j++) c[j] = __ldg(cd + grp * CW + j) * P + j;
    __syncthreads();
    const long long u = u0 + threadIdx.x;
    if (u >= nout) return;
#pragma unroll
    for (int g = 0; g < GS; g++) {
        float ftmp = 0.0f;
        for (int k = 0; k < ds; k++) {
            const float *rp = rows + (threadIdx.x * ds + k) * P;
            float acc = 0.0f;
#pragma unroll
            for (int j = 0; j < CPS; j++) acc = __fadd_rn(acc, rp[c[g * CPS + j]]);
            ftmp = __fadd_rn(ftmp, acc);
        }
        D[(long long) (grp * GS + g) * pitch + u] =
            ds == 1 ? ftmp : __fadd_rn(0.0f, __fdiv_rn(ftmp, (float) ds));
    }
}

// The same sums for any channel count: one subband per CTA, its rows staged
// one float per load (cps | 1 words apart).
__global__ void __launch_bounds__(SB_TILE) k_dd_subbands_any(const float *x, long long nspec,
                                                             int nchan, const int *cd, int cps,
                                                             int ds, long long nout,
                                                             long long pitch, int maxcd, float *D)
{
    extern __shared__ float rows[];
    __shared__ int s_cd[1024];
    const int nsub = nchan / cps;
    const int s = (int) (blockIdx.x % (unsigned) nsub);
    const int pr = cps | 1;
    const long long u0 = (long long) (blockIdx.x / (unsigned) nsub) * SB_TILE;
    const long long t_lo = u0 * ds;
    const int nrows = SB_TILE * ds + maxcd;
    for (int j = threadIdx.x; j < cps; j += blockDim.x) s_cd[j] = cd[s * cps + j];
    const float *src = x + (long long) s * cps;
    for (int e = threadIdx.x; e < nrows * cps; e += blockDim.x) {
        const int r = e / cps, j = e - r * cps;
        const long long t = t_lo + r;
        rows[r * pr + j] = t < nspec ? __ldg(src + t * nchan + j) : 0.0f;
    }
    __syncthreads();
    const long long u = u0 + threadIdx.x;
    if (u >= nout) return;
    float ftmp = 0.0f;
    for (int k = 0; k < ds; k++) {
        const int r = threadIdx.x * ds + k;
        float acc = 0.0f;
        for (int j = 0; j < cps; j++) acc = __fadd_rn(acc, rows[(r + s_cd[j]) * pr + j]);
        ftmp = __fadd_rn(ftmp, acc);
    }
    D[(long long) s * pitch + u] = ds == 1 ? ftmp : __fadd_rn(0.0f, __fdiv_rn(ftmp, (float) ds));
}

// 16-byte asynchronous copy global -> shared (both 16-byte aligned); the
// bytes past src_bytes are written as zero
__device__ __forceinline__ void cp_async16(float *dst, const float *src, int src_bytes)
{
    const unsigned d = (unsigned) __cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src),
                 "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// ints ahead of the windows in the DM stage's shared memory (16-byte rounded)
__host__ __device__ constexpr int dms_head_ints(int nsub, int g) { return (nsub * (g + 2) + 3) & ~3; }

// out[d][u] for G consecutive DMs and the DM_TILE samples of one tile;
// thread i adds samples i, i + DM_THREADS, ... (a warp's reads of a window are
// consecutive words).  blockIdx.x = sample tile * ngroups + DM group: the DM
// groups of one tile run together and share its subband rows in L2.  Per
// subband, the window of D the group reads (the tile's samples plus the
// spread of the group's offsets, from a 4-float boundary, zero past the end
// of the data) is copied into a ring of STAGES shared-memory windows by
// 16-byte asynchronous copies issued STAGES - 1 subbands ahead, so that the
// copies of later subbands are in flight while the threads add the current
// one.  D rows are pitch floats apart (a multiple of 4); wcap (a multiple of
// 4) bounds every window.
template <int G>
__global__ void __launch_bounds__(DM_THREADS) k_dd_dms(const float *D, long long nout,
                                                       long long pitch, int nsub, const int *off,
                                                       int ndm, int ngroups, int wcap, float *out)
{
    extern __shared__ __align__(16) int dsm[];
    int *s_rel = dsm;                                  // [nsub][G] offset - window start
    int *s_lo = s_rel + nsub * G;                      // [nsub] window start (a multiple of 4)
    int *s_len = s_lo + nsub;                          // [nsub] window length in 16-byte chunks
    float *win = reinterpret_cast<float *>(dsm + dms_head_ints(nsub, G));   // [STAGES][wcap]
    const int grp = (int) (blockIdx.x % (unsigned) ngroups);
    const long long u0 = (long long) (blockIdx.x / (unsigned) ngroups) * DM_TILE;
    const int d0 = grp * G;
    const int nd = min(G, ndm - d0);
    for (int s = threadIdx.x; s < nsub; s += blockDim.x) {
        int lo = off[(long long) d0 * nsub + s], hi = lo;
        for (int d = 1; d < nd; d++) {
            const int o = off[(long long) (d0 + d) * nsub + s];
            lo = min(lo, o);
            hi = max(hi, o);
        }
        lo &= ~3;
        s_lo[s] = lo;
        s_len[s] = (DM_TILE + hi - lo + 3) >> 2;
        for (int d = 0; d < G; d++)
            s_rel[s * G + d] = d < nd ? off[(long long) (d0 + d) * nsub + s] - lo : 0;
    }
    __syncthreads();
    auto issue = [&](int s) {
        if (s < nsub) {
            float *w = win + (s % STAGES) * wcap;
            const long long base = u0 + s_lo[s];
            const float *row = D + (long long) s * pitch + base;
            const long long room = nout - base;        // floats of data from the window start
            const int len4 = s_len[s];
            for (int i = threadIdx.x; i < len4; i += DM_THREADS) {
                const long long rem = room - 4LL * i;
                const int nb = rem >= 4 ? 16 : rem > 0 ? (int) rem * 4 : 0;
                cp_async16(w + 4 * i, nb > 0 ? row + 4 * i : D, nb);
            }
        }
        cp_async_commit();                             // empty groups keep the count uniform
    };
#pragma unroll
    for (int p = 0; p < STAGES - 1; p++) issue(p);
    float acc[DM_SPT][G];
#pragma unroll
    for (int k = 0; k < DM_SPT; k++)
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
            for (int k = 0; k < DM_SPT; k++) {
                acc[k][4 * q + 0] = __fadd_rn(acc[k][4 * q + 0], w[k * DM_THREADS + r.x]);
                acc[k][4 * q + 1] = __fadd_rn(acc[k][4 * q + 1], w[k * DM_THREADS + r.y]);
                acc[k][4 * q + 2] = __fadd_rn(acc[k][4 * q + 2], w[k * DM_THREADS + r.z]);
                acc[k][4 * q + 3] = __fadd_rn(acc[k][4 * q + 3], w[k * DM_THREADS + r.w]);
            }
        }
    }
    cp_async_wait<0>();
#pragma unroll
    for (int k = 0; k < DM_SPT; k++) {
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

// a window: the tile, the group's spread, up to 3 floats of alignment, in
// whole 16-byte chunks
int dms_wcap(const int *off, int ndm, int nsub, int g)
{
    return (DM_TILE + group_spread(off, ndm, nsub, g) + 3 + 3) & ~3;
}

size_t dms_smem(int g, int nsub, int wcap)
{
    return sizeof(int) * (size_t) dms_head_ints(nsub, g) + sizeof(float) * STAGES * (size_t) wcap;
}

template <int G>
cudaError_t launch_dms(const float *D, long long nout, long long pitch, int nsub, const int *off,
                       int ndm, int wcap, size_t smem, float *out, cudaStream_t st)
{
    const int ngroups = (ndm + G - 1) / G;
    const long long ntiles = (nout + DM_TILE - 1) / DM_TILE;
    if (ntiles * ngroups > 0x7FFFFFFFLL) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(k_dd_dms<G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         200 * 1024);
    if (e != cudaSuccess) return e;
    k_dd_dms<G><<<(unsigned) (ntiles * ngroups), DM_THREADS, smem, st>>>(D, nout, pitch, nsub, off,
                                                                         ndm, ngroups, wcap, out);
    return cudaGetLastError();
}

template <int CW, int CPS>
cudaError_t launch_sub(const float *x, long long nspec, int nchan, const int *cd, int ds,
                       long long nout, long long pitch, int maxcd, float *D, long long stiles,
                       cudaStream_t st)
{
    const size_t smem = sizeof(float) * (size_t) (SB_TILE * ds + maxcd) * (CW + 1);
    const long long grid = stiles * (nchan / CW);
    if (smem > 200 * 1024 || grid > 0x7FFFFFFFLL) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(k_dd_subbands<CW, CPS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess) return e;
    k_dd_subbands<CW, CPS><<<(unsigned) grid, SB_TILE, smem, st>>>(x, nspec, nchan, cd, ds, nout,
                                                                   pitch, maxcd, D);
    return cudaGetLastError();
}

cudaError_t launch_sub_any(const float *x, long long nspec, int nchan, const int *cd, int cps,
                           int ds, long long nout, long long pitch, int maxcd, float *D,
                           long long stiles, cudaStream_t st)
{
    const size_t smem = sizeof(float) * (size_t) (SB_TILE * ds + maxcd) * (size_t) (cps | 1);
    const long long grid = stiles * (nchan / cps);
    if (cps > 1024 || smem > 200 * 1024 || grid > 0x7FFFFFFFLL) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(k_dd_subbands_any,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess) return e;
    k_dd_subbands_any<<<(unsigned) grid, SB_TILE, smem, st>>>(x, nspec, nchan, cd, cps, ds, nout,
                                                              pitch, maxcd, D);
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
    if (nout < 1) return cudaErrorInvalidValue;
    const long long pitch = dedisp_sub_pitch(nout);
    const long long stiles = (nout + SB_TILE - 1) / SB_TILE;
    // DMs per thread: 16 where the trials need more than 8 and the windows
    // leave room for four CTAs per SM, else 8
    int g = ndm > 8 ? 16 : 8;
    int wcap = dms_wcap(off_host, ndm, nsub, g);
    size_t smem2 = dms_smem(g, nsub, wcap);
    if (g == 16 && smem2 > 48 * 1024) {
        g = 8;
        wcap = dms_wcap(off_host, ndm, nsub, g);
        smem2 = dms_smem(g, nsub, wcap);
    }
    if (smem2 > 200 * 1024) return cudaErrorInvalidValue;
    const bool vec = ((uintptr_t) x & 15) == 0;
    const bool w32 = vec && nchan % 32 == 0;
    cudaError_t e;
    if (w32 && cps == 1) e = launch_sub<32, 1>(x, nspec, nchan, cd, ds, nout, pitch, maxcd, D, stiles, st);
    else if (w32 && cps == 2) e = launch_sub<32, 2>(x, nspec, nchan, cd, ds, nout, pitch, maxcd, D, stiles, st);
    else if (w32 && cps == 4) e = launch_sub<32, 4>(x, nspec, nchan, cd, ds, nout, pitch, maxcd, D, stiles, st);
    else if (w32 && cps == 8) e = launch_sub<32, 8>(x, nspec, nchan, cd, ds, nout, pitch, maxcd, D, stiles, st);
    else if (w32 && cps == 16) e = launch_sub<32, 16>(x, nspec, nchan, cd, ds, nout, pitch, maxcd, D, stiles, st);
    else if (w32 && cps == 32) e = launch_sub<32, 32>(x, nspec, nchan, cd, ds, nout, pitch, maxcd, D, stiles, st);
    else if (vec && cps == 64) e = launch_sub<64, 64>(x, nspec, nchan, cd, ds, nout, pitch, maxcd, D, stiles, st);
    else e = launch_sub_any(x, nspec, nchan, cd, cps, ds, nout, pitch, maxcd, D, stiles, st);
    if (e != cudaSuccess) return e;
    return g == 16 ? launch_dms<16>(D, nout, pitch, nsub, off, ndm, wcap, smem2, out, st)
                   : launch_dms<8>(D, nout, pitch, nsub, off, ndm, wcap, smem2, out, st);
}

}  // namespace ab
