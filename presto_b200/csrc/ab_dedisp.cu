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
// row segments of a subband's channels.  The DM stage gives each thread one
// output sample of DM_GROUP consecutive DMs: nearby DMs read nearby samples
// of the same subband (the L1), and all DM groups of a sample tile run
// together (the L2 keeps the tile's subband windows).
#include <cuda_runtime.h>

#include "ab_kernels.h"

namespace ab {
namespace {

constexpr int DM_GROUP = 8;
constexpr int SB_TILE = 256;            // downsampled samples per subband CTA

// D[s][u] for u in [u0, u0 + SB_TILE) of subband s, from the time-major
// spectra x[t][c]: the rows the tile reads (its samples plus the subband's
// largest channel delay) of the subband's channels are staged in shared
// memory (each row's channels contiguous in memory, the shared rows padded to
// an odd stride so that consecutive samples hit different banks), then each
// thread sums its sample's channels and its ds samples in the reference's
// order.
__global__ void __launch_bounds__(SB_TILE) k_dd_subbands(const float *x, long long nspec, int nchan,
                                                         const int *cd, int cps, int ds,
                                                         long long nout, int maxcd, float *D)
{
    extern __shared__ float rows[];                    // [nrows][pitch]
    __shared__ int s_cd[1024];
    const int s = blockIdx.y;
    const int pitch = cps | 1;
    const long long u0 = (long long) blockIdx.x * SB_TILE;
    const long long t_lo = u0 * ds;
    const int nrows = SB_TILE * ds + maxcd;
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

// blockIdx.x = sample tile * ngroups + DM group: the DM groups of one sample
// tile run together and share its subband windows in L2
__global__ void __launch_bounds__(256) k_dd_dms(const float *D, long long nout, int nsub,
                                                const int *off, int ndm, int ngroups, float *out)
{
    extern __shared__ int s_off[];                     // [DM_GROUP][nsub]
    const int grp = (int) (blockIdx.x % (unsigned) ngroups);
    const long long tile = blockIdx.x / (unsigned) ngroups;
    const int d0 = grp * DM_GROUP;
    const int nd = min(DM_GROUP, ndm - d0);
    for (int i = threadIdx.x; i < nd * nsub; i += blockDim.x) s_off[i] = off[(long long) d0 * nsub + i];
    __syncthreads();
    const long long u = tile * blockDim.x + threadIdx.x;
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

cudaError_t launch_dedisp(const float *x, long long nspec, int nchan, const int *cd, int maxcd,
                          int nsub, int ds, const int *off, int ndm, float *D, float *out,
                          cudaStream_t st)
{
    if (nspec < 1 || nchan < 1 || nsub < 1 || nchan % nsub || ds < 1 || ndm < 1 || maxcd < 0)
        return cudaErrorInvalidValue;
    const int cps = nchan / nsub;
    const long long nout = nspec / ds;
    const size_t smem = sizeof(float) * (size_t) (SB_TILE * ds + maxcd) * (size_t) (cps | 1);
    const int ngroups = (ndm + DM_GROUP - 1) / DM_GROUP;
    const long long ntiles = (nout + 255) / 256;
    if (nout < 1 || cps > 1024 || nsub > 65535 || ntiles * ngroups > 0x7FFFFFFFLL ||
        smem > 200 * 1024)
        return cudaErrorInvalidValue;
    cudaFuncSetAttribute(k_dd_subbands, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    dim3 sg((unsigned) ((nout + SB_TILE - 1) / SB_TILE), nsub);
    k_dd_subbands<<<sg, SB_TILE, smem, st>>>(x, nspec, nchan, cd, cps, ds, nout, maxcd, D);
    k_dd_dms<<<(unsigned) (ntiles * ngroups), 256, sizeof(int) * DM_GROUP * nsub, st>>>(
        D, nout, nsub, off, ndm, ngroups, out);
    return cudaGetLastError();
}

}  // namespace ab
