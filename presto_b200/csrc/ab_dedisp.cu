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
// sample together, channels ascending in frequency); one tiled transpose puts
// each channel's samples together, so that the subband sums read
// consecutive samples per channel.  The DM stage gives each thread one
// output sample of DM_GROUP consecutive DMs: nearby DMs read nearby samples
// of the same subband, which the L1 serves.
#include <cuda_runtime.h>

#include "ab_kernels.h"

namespace ab {
namespace {

constexpr int DM_GROUP = 8;

// out (C x R) = transpose of in (R x C), 32 x 32 tiles; blockIdx.x walks the
// (long) rows, blockIdx.y the columns
__global__ void __launch_bounds__(256) k_dd_transpose(const float *in, float *out, long long R, int C)
{
    __shared__ float tile[32][33];
    const long long by = (long long) blockIdx.x * 32;
    const int bx = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += 8) {
        const long long r = by + j;
        const int c = bx + threadIdx.x;
        if (r < R && c < C) tile[j][threadIdx.x] = in[r * C + c];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int c = bx + j;
        const long long r = by + threadIdx.x;
        if (r < R && c < C) out[(long long) c * R + r] = tile[threadIdx.x][j];
    }
}

// D[s][u] from the channel-major spectra xcm[c][t]
__global__ void k_dd_subbands(const float *xcm, long long nspec, const int *cd, int cps, int ds,
                              long long nout, float *D)
{
    const long long u = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (u >= nout) return;
    float ftmp = 0.0f;
    for (int k = 0; k < ds; k++) {
        const long long t = u * ds + k;
        float acc = 0.0f;
        for (int j = 0; j < cps; j++) {
            const int c = s * cps + j;
            const long long tt = t + cd[c];
            acc = __fadd_rn(acc, tt < nspec ? __ldg(xcm + (long long) c * nspec + tt) : 0.0f);
        }
        ftmp = __fadd_rn(ftmp, acc);
    }
    D[(long long) s * nout + u] = ds == 1 ? ftmp : __fadd_rn(0.0f, __fdiv_rn(ftmp, (float) ds));
}

__global__ void __launch_bounds__(256) k_dd_dms(const float *D, long long nout, int nsub,
                                                const int *off, int ndm, float *out)
{
    extern __shared__ int s_off[];                     // [DM_GROUP][nsub]
    const int d0 = blockIdx.y * DM_GROUP;
    const int nd = min(DM_GROUP, ndm - d0);
    for (int i = threadIdx.x; i < nd * nsub; i += blockDim.x) s_off[i] = off[(long long) d0 * nsub + i];
    __syncthreads();
    const long long u = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= nout) return;
    float acc[DM_GROUP];
#pragma unroll
    for (int d = 0; d < DM_GROUP; d++) acc[d] = -0.0f;
    for (int s = 0; s < nsub; s++) {
        const float *row = D + (long long) s * nout;
#pragma unroll
        for (int d = 0; d < DM_GROUP; d++) {
            if (d < nd) {
                const long long uu = u + s_off[d * nsub + s];
                acc[d] = __fadd_rn(acc[d], uu < nout ? __ldg(row + uu) : 0.0f);
            }
        }
    }
#pragma unroll
    for (int d = 0; d < DM_GROUP; d++)
        if (d < nd) out[(long long) (d0 + d) * nout + u] = acc[d];
}

}  // namespace

cudaError_t launch_dedisp(const float *x, float *xcm, long long nspec, int nchan, const int *cd,
                          int nsub, int ds, const int *off, int ndm, float *D, float *out,
                          cudaStream_t st)
{
    if (nspec < 1 || nchan < 1 || nsub < 1 || nchan % nsub || ds < 1 || ndm < 1)
        return cudaErrorInvalidValue;
    const long long nout = nspec / ds;
    if (nout < 1 || (nspec + 31) / 32 > 0x7FFFFFFFLL || (nchan + 31) / 32 > 65535 ||
        nsub > 1024 || (ndm + DM_GROUP - 1) / DM_GROUP > 65535)
        return cudaErrorInvalidValue;
    dim3 tg((unsigned) ((nspec + 31) / 32), (nchan + 31) / 32), tb(32, 8);
    k_dd_transpose<<<tg, tb, 0, st>>>(x, xcm, nspec, nchan);
    dim3 sg((unsigned) ((nout + 255) / 256), nsub);
    k_dd_subbands<<<sg, 256, 0, st>>>(xcm, nspec, cd, nchan / nsub, ds, nout, D);
    dim3 dg((unsigned) ((nout + 255) / 256), (ndm + DM_GROUP - 1) / DM_GROUP);
    k_dd_dms<<<dg, 256, sizeof(int) * DM_GROUP * nsub, st>>>(D, nout, nsub, off, ndm, out);
    return cudaGetLastError();
}

}  // namespace ab
