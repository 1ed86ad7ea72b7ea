// ab_fft.cuh -- shared-memory FFTs for sm_100a.
//
// FP32 complex FFT of power-of-two length L in [256, 4096], Stockham
// auto-sort with radix-16 passes (plus one radix-2/4/8 pass), computed by a
// "group" of NT = L/16 threads that each hold 16 points in registers in the
// strided layout v[m] = x[t + NT*m].  A 256-thread CTA runs 4096/L groups
// side by side; every group owns (L + L/16) float2 of padded shared memory.
// Twiddles depend only on the thread, so they are computed once (FP64
// sincospi, rounded to FP32) and kept in registers across transforms.
//
// FP64 complex FFT (radix-2, in shared memory) for the one-off template
// generation.
#pragma once
#include <cuda_runtime.h>

namespace ab {

// Complex arithmetic on sm_100's paired FP32 instructions (FADD2 / FMUL2 /
// FFMA2: both components in one instruction, each rounded as the scalar
// operation would be).  a - b is fma(b, -1, a), exactly the rounded
// difference; the products keep the scalar forms' roundings:
//   a * b       = (fma(a.x, b.x, -(a.y b.y)), fma(a.x, b.y, a.y b.x))
//   a * conj(b) = (fma(a.x, b.x, a.y b.y),    fma(a.y, b.x, -(a.x b.y)))
__device__ __forceinline__ float2 operator+(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 operator-(float2 a, float2 b)
{
    return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
// a * (S i)
template <int S> __device__ __forceinline__ float2 mul_i(float2 a)
{
    return S < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}

// exp(S 2 pi i m / 16) applied to a, with the trivial angles special-cased.
template <int S, int M> __device__ __forceinline__ float2 tw16(float2 a)
{
    constexpr int m = M & 15;
    constexpr float C1 = 0.92387953251128675613f;   // cos(pi/8)
    constexpr float S1 = 0.38268343236508977173f;   // sin(pi/8)
    constexpr float H = 0.70710678118654752440f;    // cos(pi/4)
    if constexpr (m == 0) {
        return a;
    } else if constexpr (m == 4) {
        return mul_i<S>(a);
    } else if constexpr (m == 8) {
        return make_float2(-a.x, -a.y);
    } else if constexpr (m == 12) {
        return mul_i<-S>(a);
    } else if constexpr (m == 2 || m == 6 || m == 10 || m == 14) {
        // (+-1 +- i) H
        constexpr float cr = (m == 2 || m == 14) ? H : -H;
        constexpr float ci = ((m == 2 || m == 6) ? H : -H) * (S < 0 ? -1.f : 1.f);
        return cmul(a, make_float2(cr, ci));
    } else {
        constexpr float cr = (m == 1 || m == 15) ? C1 : (m == 3 || m == 13) ? S1
                           : (m == 5 || m == 11) ? -S1 : -C1;
        constexpr float si = (m == 1 || m == 7) ? S1 : (m == 3 || m == 5) ? C1
                           : (m == 9 || m == 15) ? -S1 : -C1;
        constexpr float ci = si * (S < 0 ? -1.f : 1.f);
        return cmul(a, make_float2(cr, ci));
    }
}

template <int S> __device__ __forceinline__ void dft2(float2 *x)
{
    float2 t = x[0];
    x[0] = t + x[1];
    x[1] = t - x[1];
}

template <int S> __device__ __forceinline__ void dft4v(float2 &a0, float2 &a1, float2 &a2, float2 &a3)
{
    const float2 t0 = a0 + a2, t1 = a0 - a2, t2 = a1 + a3, d = a1 - a3;
    a0 = t0 + t2;
    a2 = t0 - t2;
    // t1 +- (S i) d: cross-component sums, as scalar operations
    if constexpr (S < 0) {
        a1 = make_float2(t1.x + d.y, t1.y - d.x);
        a3 = make_float2(t1.x - d.y, t1.y + d.x);
    } else {
        a1 = make_float2(t1.x - d.y, t1.y + d.x);
        a3 = make_float2(t1.x + d.y, t1.y - d.x);
    }
}

template <int S> __device__ __forceinline__ void dft4(float2 *x) { dft4v<S>(x[0], x[1], x[2], x[3]); }

template <int S> __device__ __forceinline__ void dft8(float2 *x)
{
    dft4v<S>(x[0], x[2], x[4], x[6]);
    dft4v<S>(x[1], x[3], x[5], x[7]);
    float2 o1 = tw16<S, 2>(x[3]), o2 = tw16<S, 4>(x[5]), o3 = tw16<S, 6>(x[7]);
    float2 e0 = x[0], e1 = x[2], e2 = x[4], e3 = x[6], o0 = x[1];
    x[0] = e0 + o0; x[4] = e0 - o0;
    x[1] = e1 + o1; x[5] = e1 - o1;
    x[2] = e2 + o2; x[6] = e2 - o2;
    x[3] = e3 + o3; x[7] = e3 - o3;
}

template <int S> __device__ __forceinline__ void dft16(float2 *x)
{
    // n = 4 n1 + n2, k = k1 + 4 k2
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) dft4v<S>(x[n2], x[4 + n2], x[8 + n2], x[12 + n2]);
    // x[n2 + 4 k1] = A[n2][k1]; twiddle by w16^(n2 k1)
    x[5] = tw16<S, 1>(x[5]);
    x[9] = tw16<S, 2>(x[9]);
    x[13] = tw16<S, 3>(x[13]);
    x[6] = tw16<S, 2>(x[6]);
    x[10] = tw16<S, 4>(x[10]);
    x[14] = tw16<S, 6>(x[14]);
    x[7] = tw16<S, 3>(x[7]);
    x[11] = tw16<S, 6>(x[11]);
    x[15] = tw16<S, 9>(x[15]);
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) dft4v<S>(x[4 * k1], x[4 * k1 + 1], x[4 * k1 + 2], x[4 * k1 + 3]);
    // x[4 k1 + k2] = X[k1 + 4 k2]  -> natural order
    float2 y[16];
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++)
#pragma unroll
        for (int k2 = 0; k2 < 4; k2++) y[k1 + 4 * k2] = x[4 * k1 + k2];
#pragma unroll
    for (int i = 0; i < 16; i++) x[i] = y[i];
}

template <int R, int S> __device__ __forceinline__ void dft(float2 *x)
{
    if constexpr (R == 2) dft2<S>(x);
    else if constexpr (R == 4) dft4<S>(x);
    else if constexpr (R == 8) dft8<S>(x);
    else dft16<S>(x);
}

__device__ __forceinline__ int pad16(int i) { return i + (i >> 4); }

template <int L> struct FftShape {
    static constexpr int NT = L / 16;                 // threads per transform
    static constexpr int CTA = NT > 256 ? NT : 256;   // threads per CTA
    static constexpr int G = CTA / NT;                // transforms per CTA
    static constexpr int MINB = CTA <= 256 ? 2 : 1;   // CTAs per SM the register cap keeps
    static constexpr int R3 = L <= 4096 ? L / 256 : 16;   // radix of the third pass (1: none)
    static constexpr int R4 = L > 4096 ? L / 4096 : 1;    // radix of the fourth pass (1: none)
    static constexpr int NB3 = (R3 > 1) ? 16 / R3 : 0;
    static constexpr int NB4 = (R4 > 1) ? 16 / R4 : 0;
    static constexpr int SMEM = L + L / 16;           // padded float2 per transform
    // shared-memory exchanges per transform (passes - 1); with exactly two,
    // a second buffer removes the barrier after each read-back (DBUF)
    static constexpr int NEX = 1 + (R3 > 1 ? 1 : 0) + (R4 > 1 ? 1 : 0);
    static constexpr bool DBUF = NEX == 2;
    static_assert(L >= 256 && L <= 8192 && (L & (L - 1)) == 0, "FFT length");
};

// Per-thread twiddles of passes 2, 3 and 4 (pass 1 has none), stored as the
// base powers w, w^2, w^4, w^8 of each butterfly's root w; the other powers
// are formed with at most three complex products (a few ulp of error).
template <int L, int S> struct FftTw {
    using SH = FftShape<L>;
    static constexpr int NBASE3 = SH::R3 >= 16 ? 4 : SH::R3 >= 8 ? 3 : SH::R3 >= 4 ? 2 : 1;
    float2 b2[4];                                   // pass 2: w = exp(S 2 pi i k / 256)
    float2 b3[SH::NB3 > 0 ? SH::NB3 : 1][NBASE3];   // pass 3: w = exp(S 2 pi i k / (256 R3))
    float2 b4[SH::NB4 > 0 ? SH::NB4 : 1];           // pass 4 (radix 2): w = exp(S 2 pi i k / L)
    __device__ __forceinline__ void init(int t)
    {
        int k = t & 15;
#pragma unroll
        for (int e = 0; e < 4; e++) {
            double s, c;
            sincospi(2.0 * (double) (k << e) / 256.0, &s, &c);
            b2[e] = make_float2((float) c, (float) (S * s));
        }
        if constexpr (SH::R3 > 1) {
#pragma unroll
            for (int b = 0; b < SH::NB3; b++) {
                int kk = (t + SH::NT * b) & 255;
#pragma unroll
                for (int e = 0; e < NBASE3; e++) {
                    double s, c;
                    sincospi(2.0 * (double) (kk << e) / (double) (256 * SH::R3), &s, &c);
                    b3[b][e] = make_float2((float) c, (float) (S * s));
                }
            }
        }
        if constexpr (SH::R4 > 1) {
            static_assert(SH::R4 == 2, "fourth pass is radix 2");
#pragma unroll
            for (int b = 0; b < SH::NB4; b++) {
                int kk = (t + SH::NT * b) & 4095;
                double s, c;
                sincospi(2.0 * (double) kk / (double) L, &s, &c);
                b4[b] = make_float2((float) c, (float) (S * s));
            }
        }
    }
};

// x[q] *= w^q for q = 1..R-1, w^q built from the base powers.
template <int R>
__device__ __forceinline__ void apply_tw(float2 *x, const float2 *bs)
{
    if constexpr (R >= 2) x[1] = cmul(x[1], bs[0]);
    if constexpr (R >= 4) {
        x[2] = cmul(x[2], bs[1]);
        float2 p3 = cmul(bs[1], bs[0]);
        x[3] = cmul(x[3], p3);
        if constexpr (R >= 8) {
            x[4] = cmul(x[4], bs[2]);
            float2 p5 = cmul(bs[2], bs[0]), p6 = cmul(bs[2], bs[1]), p7 = cmul(p6, bs[0]);
            x[5] = cmul(x[5], p5);
            x[6] = cmul(x[6], p6);
            x[7] = cmul(x[7], p7);
            if constexpr (R >= 16) {
                x[8] = cmul(x[8], bs[3]);
                float2 p9 = cmul(bs[3], bs[0]), p10 = cmul(bs[3], bs[1]), p12 = cmul(bs[3], bs[2]);
                x[9] = cmul(x[9], p9);
                x[10] = cmul(x[10], p10);
                x[11] = cmul(x[11], cmul(p10, bs[0]));
                x[12] = cmul(x[12], p12);
                x[13] = cmul(x[13], cmul(p12, bs[0]));
                float2 p14 = cmul(p12, bs[1]);
                x[14] = cmul(x[14], p14);
                x[15] = cmul(x[15], cmul(p14, bs[0]));
            }
        }
    }
}

template <int L, int S, int PASS>
__device__ __forceinline__ void apply_tw_pass(float2 *x, int b, int t, const FftTw<L, S> &tw)
{
    if constexpr (PASS == 2) apply_tw<16>(x, tw.b2);
    if constexpr (PASS == 3) apply_tw<FftShape<L>::R3>(x, tw.b3[b]);
    if constexpr (PASS == 4) apply_tw<FftShape<L>::R4>(x, &tw.b4[b]);
}

// One Stockham pass.  v holds x[t + NT m]; results of a non-final pass go
// through shared memory and come back in the same strided layout.
// PASS: 1 to 4 (selects the twiddles).  TW: FftTw (register bases).
// TRAIL: barrier after the read-back (not needed when the next exchange
// writes another buffer).
template <int L, int R, int LS, int S, bool LAST, int PASS, bool TRAIL = true, class TW>
__device__ __forceinline__ void fft_pass(float2 (&v)[16], float2 *sm, int t, const TW &tw)
{
    constexpr int NT = L / 16, NB = 16 / R;
#pragma unroll
    for (int b = 0; b < NB; b++) {
        float2 x[R];
#pragma unroll
        for (int q = 0; q < R; q++) x[q] = v[b + q * NB];
        if constexpr (PASS > 1) apply_tw_pass<L, S, PASS>(x, b, t, tw);
        dft<R, S>(x);
        if constexpr (LAST) {
#pragma unroll
            for (int s = 0; s < R; s++) v[b + s * NB] = x[s];
        } else {
            int j = t + NT * b;
            int k = j & (LS - 1);
            int base = (j - k) * R + k;
#pragma unroll
            for (int s = 0; s < R; s++) sm[pad16(base + s * LS)] = x[s];
        }
    }
    if constexpr (!LAST) {
        __syncthreads();
#pragma unroll
        for (int m = 0; m < 16; m++) v[m] = sm[pad16(t + NT * m)];
        if constexpr (TRAIL) __syncthreads();
    }
}

// Full transform of the group's data, in place in v.  Must be called by all
// threads of the CTA (it contains __syncthreads).  With sm2 (a second
// buffer of SMEM float2, only where FftShape<L>::DBUF) the two exchanges use
// sm then sm2 and skip the barrier after each read-back: a buffer is written
// again only after every thread has passed the barrier of the other
// exchange, which follows its last read of that buffer.
template <int L, int S, class TW>
__device__ __forceinline__ void fft_run(float2 (&v)[16], float2 *sm, int t, const TW &tw,
                                        float2 *sm2 = nullptr)
{
    using SH = FftShape<L>;
    if constexpr (SH::DBUF) {
        if (sm2) {
            fft_pass<L, 16, 1, S, false, 1, false>(v, sm, t, tw);
            fft_pass<L, 16, 16, S, false, 2, false>(v, sm2, t, tw);
            fft_pass<L, SH::R3, 256, S, true, 3>(v, sm, t, tw);
            return;
        }
    }
    if constexpr (SH::R4 > 1) {
        fft_pass<L, 16, 1, S, false, 1>(v, sm, t, tw);
        fft_pass<L, 16, 16, S, false, 2>(v, sm, t, tw);
        fft_pass<L, 16, 256, S, false, 3>(v, sm, t, tw);
        fft_pass<L, SH::R4, 4096, S, true, 4>(v, sm, t, tw);
    } else if constexpr (SH::R3 > 1) {
        fft_pass<L, 16, 1, S, false, 1>(v, sm, t, tw);
        fft_pass<L, 16, 16, S, false, 2>(v, sm, t, tw);
        fft_pass<L, SH::R3, 256, S, true, 3>(v, sm, t, tw);
    } else {
        fft_pass<L, 16, 1, S, false, 1>(v, sm, t, tw);
        fft_pass<L, 16, 16, S, true, 2>(v, sm, t, tw);
    }
}

// ---------------------------------------------------------------------
// FP64 radix-2 FFT in shared memory (templates).  tw[m] = exp(S 2 pi i m/n)
// for m < n/2 (global table).  All threads of the CTA call it.
// ---------------------------------------------------------------------
__device__ __forceinline__ double2 dmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

static __device__ void fft64_inplace(double2 *x, int n, int log2n, const double2 *tw)
{
    // bit reversal
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        int j = __brev(i) >> (32 - log2n);
        if (j > i) {
            double2 a = x[i];
            x[i] = x[j];
            x[j] = a;
        }
    }
    __syncthreads();
    for (int half = 1, st = n >> 1; half < n; half <<= 1, st >>= 1) {
        for (int b = threadIdx.x; b < n / 2; b += blockDim.x) {
            int grp = b / half, k = b - grp * half;
            int i0 = grp * 2 * half + k, i1 = i0 + half;
            double2 w = tw[k * st];
            double2 u = x[i0], v = dmul(x[i1], w);
            x[i0] = make_double2(u.x + v.x, u.y + v.y);
            x[i1] = make_double2(u.x - v.x, u.y - v.y);
        }
        __syncthreads();
    }
}

}  // namespace ab
