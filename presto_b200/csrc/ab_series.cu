// ab_series.cu -- the time-series input path of the search on the device:
// create_accelobs' .dat branch (src/accel_utils.c:1516-1563), i.e. the
// forward realfft (src/fastffts.c:163-246) and deredden(fft, n/2, 6, 200,
// 0.5/dt, n dt) (src/misc_utils.c:912-1067).
//
// realfft: the n/2-point complex FFT of the samples taken in pairs, then the
// untangling pass into n/2 bins with bin 0 = (DC, Nyquist).  For a
// power-of-two M = n/2 the complex FFT is one radix-16 Stockham transform in
// shared memory up to 8192 points, and above that a four-step transform
// M = M1 M2: transpose, M2 transforms of length M1 multiplied by
// exp(-2 pi i n2 k1 / M), transpose, M1 transforms of length M2, transpose
// (each step one pass over HBM).  Any other even n (dedispersed series are
// usually 2^a 3^b 5^c 7^d samples long) goes through Bluestein's chirp-z
// transform on three power-of-two transforms of length >= 2M - 1.
//
// deredden: the block partition depends only on bin indices (lengths
// startwidth ln(bin) up to endwidth), so the host plans it; one CTA per block
// takes the exact median of its powers, then one CTA per segment between
// block midpoints scales the bins by the reference's interpolated
// normalisation with its fast inverse square root, in float with explicit
// rounding, so the same input gives the reference's bits.
#include <cuda_runtime.h>
#include <math.h>

#include "ab_fft.cuh"
#include "ab_kernels.h"
#include "ab_norm.cuh"
#include "ab_select.cuh"

namespace ab {
namespace {

template <int L>
__global__ void __launch_bounds__(FftShape<L>::CTA) k_fft_rows(const float2 *in, float2 *out,
                                                             long long rows, long long twM)
{
    using SH = FftShape<L>;
    extern __shared__ float2 fsm[];
    const int grp = threadIdx.x / SH::NT, t = threadIdx.x - grp * SH::NT;
    const long long row = (long long) blockIdx.x * SH::G + grp;
    float2 *sm = fsm + grp * SH::SMEM;
    FftTw<L, -1> tw;
    tw.init(t);
    const bool ok = row < rows;
    float2 v[16];
#pragma unroll
    for (int m = 0; m < 16; m++) v[m] = ok ? in[row * L + t + SH::NT * m] : make_float2(0.f, 0.f);
    fft_run<L, -1>(v, sm, t, tw);
    if (!ok) return;
#pragma unroll
    for (int m = 0; m < 16; m++) {
        const long long k = t + SH::NT * m;
        float2 y = v[m];
        if (twM) {
            // W_M^{row k} = exp(-2 pi i row k / M), argument reduced mod M
            double s, c;
            sincospi(-2.0 * (double) ((row * k) % twM) / (double) twM, &s, &c);
            const float cr = (float) c, ci = (float) s;
            y = make_float2(y.x * cr - y.y * ci, y.x * ci + y.y * cr);
        }
        out[row * L + k] = y;
    }
}

// out (C x R) = transpose of in (R x C), 32 x 32 tiles
__global__ void __launch_bounds__(256) k_transpose(const float2 *in, float2 *out, int R, int C)
{
    __shared__ float2 tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int r = by + j, c = bx + threadIdx.x;
        if (r < R && c < C) tile[j][threadIdx.x] = in[(long long) r * C + c];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int c = bx + j, r = by + threadIdx.x;
        if (r < R && c < C) out[(long long) c * R + r] = tile[threadIdx.x][j];
    }
}

// realfft's untangling (src/fastffts.c:195-229, forward): pair (il, n/2 - il)
// per thread, sums of the float inputs in float as the reference, products
// in FP64 without contraction, twiddles exp(-2 pi i il / n) computed directly.
__global__ void k_untangle(float2 *c, long long n)
{
    const long long il = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    const long long nby2 = n >> 1, nby4 = n >> 2;
    if (il == 0) {
        const float t = c[0].x;
        c[0] = make_float2(__fadd_rn(t, c[0].y), __fsub_rn(t, c[0].y));
        return;
    }
    if (il > nby4) return;
    const long long ih = nby2 - il;
    const float2 a = c[il], b = c[ih];
    double wi, wr;
    sincospi(-2.0 * (double) il / (double) n, &wi, &wr);
    const double h1r = 0.5 * (double) __fadd_rn(a.x, b.x), h1i = 0.5 * (double) __fsub_rn(a.y, b.y);
    const double h2r = 0.5 * (double) __fadd_rn(a.y, b.y), h2i = -0.5 * (double) __fsub_rn(a.x, b.x);
    const double h2rwr = __dmul_rn(h2r, wr), h2rwi = __dmul_rn(h2r, wi);
    const double h2iwr = __dmul_rn(h2i, wr), h2iwi = __dmul_rn(h2i, wi);
    const float2 lo = make_float2((float) __dsub_rn(__dadd_rn(h1r, h2rwr), h2iwi),
                                  (float) __dadd_rn(__dadd_rn(h1i, h2iwr), h2rwi));
    const float2 hi = make_float2((float) __dadd_rn(__dsub_rn(h1r, h2rwr), h2iwi),
                                  (float) __dadd_rn(__dadd_rn(-h1i, h2iwr), h2rwi));
    c[il] = lo;
    c[ih] = hi;
}


// Median of each block's powers / ln 2 (the block "mean" of deredden), one
// 32-thread CTA per block.
__global__ void __launch_bounds__(32) k_dered_means(const float2 *fft, const int2 *blocks, float *means)
{
    __shared__ float pw[AB_DERED_MAXW];
    __shared__ unsigned hist[256], res[2];
    const int2 b = blocks[blockIdx.x];
    for (int i = threadIdx.x; i < b.y; i += blockDim.x) {
        const float2 v = fft[b.x + i];
        pw[i] = __fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y));
    }
    __syncthreads();
    const float lo = select_rank(pw, b.y, (b.y - 1) / 2, hist, res);
    const float hi = (b.y & 1) ? lo : select_rank(pw, b.y, b.y / 2, hist, res);
    if (threadIdx.x == 0) {
        const float med = (b.y & 1) ? lo : (float) (0.5 * ((double) lo + (double) hi));
        means[blockIdx.x] = (float) ((double) med / 0.69314718055994530942);
    }
}

// Segment s of the output (one CTA each): s = 0 is the first half of block 0
// (no slope); s = 1..nb-1 runs from the midpoint of block s-1 to the midpoint
// of block s with the slope between their means; s = nb is the second half
// of the last block with the last slope (1 when there is one block).  Bin 0
// becomes (1, 0).
__global__ void __launch_bounds__(256) k_dered_apply(float2 *fft, const int2 *blocks, const float *means,
                                                    int nb)
{
    const int s = blockIdx.x;
    long long start, end;
    float mean_old, dslope = 1.0f;
    if (s == 0) {
        start = blocks[0].x;
        end = start + blocks[0].y / 2;
        mean_old = means[0];
        if (threadIdx.x == 0) fft[0] = make_float2(1.0f, 0.0f);
    } else {
        const int k = s < nb ? s : nb - 1;              // slope of blocks k-1, k
        if (k >= 1) {
            const int2 b0 = blocks[k - 1], b1 = blocks[k];
            dslope = (float) ((double) __fsub_rn(means[k], means[k - 1]) / (0.5 * (double) (b0.y + b1.y)));
        }
        const int2 bo = blocks[s - 1];
        start = bo.x + bo.y / 2;
        end = (s < nb) ? blocks[s].x + blocks[s].y / 2 : bo.x + bo.y;
        mean_old = means[s - 1];
    }
    for (long long bin = start + threadIdx.x; bin < end; bin += blockDim.x) {
        const float ii = (float) (bin - start);
        const float norm = (s == 0) ? fast_invsqrtf(mean_old)
                                    : fast_invsqrtf(__fadd_rn(mean_old, __fmul_rn(dslope, ii)));
        const float2 v = fft[bin];
        fft[bin] = make_float2(__fmul_rn(v.x, norm), __fmul_rn(v.y, norm));
    }
}

template <int L>
cudaError_t fft_rows_L(const float2 *in, float2 *out, long long rows, long long twM, cudaStream_t st)
{
    using SH = FftShape<L>;
    const size_t smem = (size_t) SH::G * SH::SMEM * sizeof(float2);
    cudaFuncSetAttribute(k_fft_rows<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    const long long grid = (rows + SH::G - 1) / SH::G;
    k_fft_rows<L><<<(unsigned) grid, SH::CTA, smem, st>>>(in, out, rows, twM);
    return cudaGetLastError();
}

cudaError_t fft_rows(int L, const float2 *in, float2 *out, long long rows, long long twM, cudaStream_t st)
{
    switch (L) {
        case 256: return fft_rows_L<256>(in, out, rows, twM, st);
        case 512: return fft_rows_L<512>(in, out, rows, twM, st);
        case 1024: return fft_rows_L<1024>(in, out, rows, twM, st);
        case 2048: return fft_rows_L<2048>(in, out, rows, twM, st);
        case 4096: return fft_rows_L<4096>(in, out, rows, twM, st);
        case 8192: return fft_rows_L<8192>(in, out, rows, twM, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t transpose(const float2 *in, float2 *out, int R, int C, cudaStream_t st)
{
    dim3 grid((C + 31) / 32, (R + 31) / 32), block(32, 8);
    k_transpose<<<grid, block, 0, st>>>(in, out, R, C);
    return cudaGetLastError();
}

// Forward complex FFT of M points, M a power of two in 512..8192 or 2^16..2^26;
// out may be in, scratch (M points) may not.
cudaError_t cfft_pow2(const float2 *in, float2 *out, float2 *scratch, long long M, cudaStream_t st)
{
    if (M <= 8192) return fft_rows((int) M, in, out, 1, 0, st);
    int m = 0;
    while ((1LL << m) < M) m++;
    const int M1 = 1 << (m / 2), M2 = (int) (M / M1);
    // x[n1][n2] (M1 x M2) -> scratch[n2][n1]; rows of length M1 with the
    // twiddle; -> out[k1][n2]; rows of length M2; -> scratch[k2][k1]; copy
    cudaError_t e = transpose(in, scratch, M1, M2, st);
    if (e == cudaSuccess) e = fft_rows(M1, scratch, scratch, M2, M, st);
    if (e == cudaSuccess) e = transpose(scratch, out, M2, M1, st);
    if (e == cudaSuccess) e = fft_rows(M2, out, out, M1, 0, st);
    if (e == cudaSuccess) e = transpose(out, scratch, M1, M2, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, scratch, sizeof(float2) * M, cudaMemcpyDeviceToDevice, st);
    return e;
}

// Bluestein's chirp-z transform for any length M: with c_j = exp(i pi j^2 / M),
// X_k = conj(c_k) sum_j (x_j conj(c_j)) c_{k-j}, a linear convolution done as
// a circular one of power-of-two length L >= 2M - 1.  Chirps are evaluated in
// FP64 from j^2 mod 2M (exact in 64-bit integers), the products with them in
// FP64; the three length-L transforms are the FP32 power-of-two FFT above.
__device__ __forceinline__ void chirp(long long j, long long M, double &c, double &s)
{
    const long long r = (j * j) % (2 * M);
    sincospi((double) r / (double) M, &s, &c);
}

__global__ void k_blu_pre(const float2 *z, float2 *a, long long M, long long L)
{
    const long long j = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= L) return;
    if (j >= M) {
        a[j] = make_float2(0.f, 0.f);
        return;
    }
    double c, s;
    chirp(j, M, c, s);
    const double xr = z[j].x, xi = z[j].y;           // x conj(c)
    a[j] = make_float2((float) (xr * c + xi * s), (float) (xi * c - xr * s));
}

__global__ void k_blu_kernel(float2 *b, long long M, long long L)
{
    const long long j = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= L) return;
    const long long m = j < M ? j : (j > L - M ? L - j : -1);
    if (m < 0) {
        b[j] = make_float2(0.f, 0.f);
        return;
    }
    double c, s;
    chirp(m, M, c, s);
    b[j] = make_float2((float) c, (float) s);
}

// a = conj(a B): the inverse transform as a forward one of the conjugate
__global__ void k_blu_mul(float2 *a, const float2 *B, long long L)
{
    const long long j = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= L) return;
    const float2 x = a[j], y = B[j];
    a[j] = make_float2(x.x * y.x - x.y * y.y, -(x.x * y.y + x.y * y.x));
}

__global__ void k_blu_post(const float2 *v, float2 *out, long long M, long long L)
{
    const long long k = (long long) blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M) return;
    double c, s;
    chirp(k, M, c, s);
    const double inv = 1.0 / (double) L;
    const double yr = (double) v[k].x * inv, yi = -(double) v[k].y * inv;   // conj(v) / L
    out[k] = make_float2((float) (yr * c + yi * s), (float) (yi * c - yr * s));
}

}  // namespace

bool pow2_fft_supported(long long M)
{
    if (M & (M - 1)) return false;
    return (M >= 512 && M <= 8192) || (M >= (1 << 16) && M <= (1LL << 26));
}

long long bluestein_len(long long M)
{
    long long L = 1;
    while (L < 2 * M - 1) L <<= 1;
    if (L < 512) L = 512;
    if (L > 8192 && L < (1 << 16)) L = 1 << 16;       // the four-step's shortest
    return L;
}

bool realfft_supported(long long n)
{
    if (n < 1024 || n % 2) return false;
    const long long M = n / 2;
    return pow2_fft_supported(M) || M <= (1LL << 25);
}

cudaError_t launch_realfft(const float *series, float2 *out, float2 *scratch, long long n, cudaStream_t st)
{
    const long long M = n / 2;
    if (n % 2 || !pow2_fft_supported(M)) return cudaErrorInvalidValue;
    cudaError_t e = cfft_pow2(reinterpret_cast<const float2 *>(series), out, scratch, M, st);
    if (e != cudaSuccess) return e;
    const long long nthr = M / 2 + 1;
    k_untangle<<<(unsigned) ((nthr + 255) / 256), 256, 0, st>>>(out, n);
    return cudaGetLastError();
}

cudaError_t launch_realfft_bluestein(const float *series, float2 *out, float2 *a, float2 *scratch,
                                     float2 *B, bool build_B, long long n, cudaStream_t st)
{
    const long long M = n / 2, L = bluestein_len(M);
    if (n % 2 || n < 1024 || M > (1LL << 25)) return cudaErrorInvalidValue;
    const unsigned gL = (unsigned) ((L + 255) / 256), gM = (unsigned) ((M + 255) / 256);
    cudaError_t e = cudaSuccess;
    if (build_B) {                                   // FFT of the chirp kernel, kept per M
        k_blu_kernel<<<gL, 256, 0, st>>>(B, M, L);
        e = cfft_pow2(B, B, scratch, L, st);
        if (e != cudaSuccess) return e;
    }
    k_blu_pre<<<gL, 256, 0, st>>>(reinterpret_cast<const float2 *>(series), a, M, L);
    e = cfft_pow2(a, a, scratch, L, st);
    if (e != cudaSuccess) return e;
    k_blu_mul<<<gL, 256, 0, st>>>(a, B, L);
    e = cfft_pow2(a, a, scratch, L, st);
    if (e != cudaSuccess) return e;
    k_blu_post<<<gM, 256, 0, st>>>(a, out, M, L);
    const long long nthr = M / 2 + 1;
    k_untangle<<<(unsigned) ((nthr + 255) / 256), 256, 0, st>>>(out, n);
    return cudaGetLastError();
}

cudaError_t launch_deredden(float2 *fft, const int2 *blocks, int nb, float *means, cudaStream_t st)
{
    if (nb <= 0) return cudaErrorInvalidValue;
    k_dered_means<<<nb, 32, 0, st>>>(fft, blocks, means);
    k_dered_apply<<<nb + 1, 256, 0, st>>>(fft, blocks, means, nb);
    return cudaGetLastError();
}

}  // namespace ab
