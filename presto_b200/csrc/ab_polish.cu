// ab_polish.cu -- candidate polishing on the device: optimize_accelcand
// (src/accel_utils.c:552-626) for acceleration searches with harmonic
// polishing, the reference's default, every candidate of a search at once.
//
// One CTA of 256 threads per candidate runs max_rz_arr_harmonics
// (src/maximize_rz.c:173-228): local powers of the harmonics, two
// Nelder-Mead stages over (r, z / 4) maximising the sum of the harmonics'
// locally normalised powers (LOWACC kernels, step 0.4, size tolerance 1e-4;
// then HIGHACC kernels, step 0.01, 1e-7), then each harmonic's power, local
// power and derivatives (get_localpower3d, get_derivs3d,
// src/characteristics.c:79-193).  Complex amplitudes at fractional (r, z)
// come from rz_interp (src/rzinterp.c:144-232): a warp correlates the data
// with the FP64 response generated at the fractional offset, lanes splitting
// the kernel points.  The simplex bookkeeping runs identically in every
// thread; each function value is reduced by thread 0 in the reference's
// harmonic order and broadcast through shared memory, so control flow stays
// uniform.  Iterations are bounded (5000 per stage, as the reference).
#include <cuda_runtime.h>
#include <math.h>

#include "ab_kernels.h"
#include "ab_resp.cuh"

namespace ab {
namespace {

constexpr int PL_THREADS = 512;
constexpr int PL_WARPS = PL_THREADS / 32;
constexpr int PL_MAXH = AB_POLISH_MAX_HARM;
constexpr int PL_LOCPOW = 20;                 // NUMLOCPOWAVG, include/presto.h:99
constexpr int PL_DELTA = 5;                   // DELTAAVGBINS, include/presto.h:103
constexpr double PL_ZSCALE = 4.0;             // src/maximize_rz.c:6
constexpr int PL_ITEMS = PL_MAXH * PL_LOCPOW;

__device__ __forceinline__ int z_halfwidth(double z, bool highacc)   // src/responses.c:27-47
{
    return (int) (0.5 * 1.1 * fabs(z)) + (highacc ? 48 : 16);
}

// rz_interp (src/rzinterp.c:144-232) at (r, z) with kernel half-width hw,
// shared by P warps: this lane of warp part sums kernel points lane + 32 (part
// + P k) in FP64.  The lanes' and parts' sums add up to the amplitude; the
// exact-bin cases come from lane 0 of part 0 alone.
__device__ double2 rz_interp_part(const float2 *data, long long numdata, double r, double z, int hw,
                                  int part, int P, int lane)
{
    if (r > numdata - 1.0 || r < 0.0) return make_double2(0.0, 0.0);
    double dint;
    const double frac = modf(r, &dint);
    const long long intfreq = (long long) dint;
    if (fabs(z) < 1E-4) {
        const bool first = part == 0 && lane == 0;
        if (frac < 1E-5) {
            const float2 v = data[intfreq];
            return first ? make_double2(v.x, v.y) : make_double2(0.0, 0.0);
        }
        if ((1.0 - frac) < 1E-5) {
            const float2 v = data[intfreq + 1];
            return first ? make_double2(v.x, v.y) : make_double2(0.0, 0.0);
        }
    }
    const int numkern = 2 * hw;
    long long lodata = intfreq - hw, loresp = 0;
    if (lodata < 0) {
        loresp = -lodata;
        lodata = 0;
    }
    const long long hidata = intfreq + hw - 1;
    const long long hiresp = (hidata > numdata - 1) ? numkern - hidata + numdata - 1 : numkern;
    const long long nsum = hiresp - loresp;
    double ar = 0.0, ai = 0.0;
    for (long long ii = lane + 32 * part; ii < nsum; ii += 32 * P) {
        const double2 pv = z_resp_point(frac, 1, z, numkern, (int) (loresp + ii));
        const float pr = (float) pv.x, pim = (float) pv.y;      // the reference's response is float
        const float2 d = data[lodata + ii];
        ar += (double) d.x * (double) pr + (double) __fmul_rn(d.y, pim);
        ai += (double) d.y * (double) pr - (double) pim * (double) d.x;
    }
    return make_double2(ar, ai);
}

__device__ __forceinline__ double2 warp_sum(double2 v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}

// rz_interp by one warp.
__device__ float2 warp_rz_interp(const float2 *data, long long numdata, double r, double z, int hw,
                                 int lane)
{
    const double2 v = warp_sum(rz_interp_part(data, numdata, r, z, hw, 0, 1, lane));
    return make_float2((float) v.x, (float) v.y);
}

__device__ __forceinline__ double powerf2(float2 a) { return (double) a.x * a.x + (double) a.y * a.y; }

struct PolishSmem {
    double r[PL_ITEMS], z[PL_ITEMS];
    int hw[PL_ITEMS];
    float2 amp[PL_ITEMS];
    int cnt[PL_MAXH];
    double term[PL_MAXH];
    float locpow[PL_MAXH];
    double2 part[PL_MAXH];      // per-warp partial amplitudes of one evaluation
    double val;
    int raw;                    // max_rz_arr: one harmonic, raw power (-noharmpolish)
};

// Amplitudes of items [0, n) (all threads).
__device__ void interp_items(const float2 *data, long long numdata, int n, PolishSmem &s)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int it = warp; it < n; it += PL_WARPS) {
        const float2 a = warp_rz_interp(data, numdata, s.r[it], s.z[it], s.hw[it], lane);
        if (lane == 0) s.amp[it] = a;
    }
    __syncthreads();
}

// get_localpower3d (w = 0) of harmonic n = 1..nh at (r n, z n) into s.locpow
// (float, as max_rz_arr_harmonics keeps them).
__device__ void local_powers(const float2 *data, long long numdata, double r, double z, int nh,
                             PolishSmem &s)
{
    if (threadIdx.x == 0) {
        int k = 0;
        for (int ii = 0; ii < nh; ii++) {
            const double rh = r * (ii + 1), zh = z * (ii + 1);
            const int hw = z_halfwidth(zh, false);
            double lo1 = rh - PL_DELTA - PL_LOCPOW / 2, hi1 = lo1 + PL_LOCPOW / 2;
            double lo2 = rh + PL_DELTA, hi2 = lo2 + PL_LOCPOW / 2;
            double *b[4] = {&lo1, &lo2, &hi1, &hi2};
            for (int q = 0; q < 4; q++) {
                if (*b[q] < 0.0) *b[q] = 0.0;
                if (*b[q] > numdata) *b[q] = (double) numdata;
            }
            int c = 0;
            for (double f = lo1; f < hi1 && k < PL_ITEMS; f += 1.0, c++, k++) {
                s.r[k] = f;
                s.z[k] = zh;
                s.hw[k] = hw;
            }
            for (double f = lo2; f < hi2 && k < PL_ITEMS; f += 1.0, c++, k++) {
                s.r[k] = f;
                s.z[k] = zh;
                s.hw[k] = hw;
            }
            s.cnt[ii] = c;
        }
        s.val = (double) k;
    }
    __syncthreads();
    const int n = (int) s.val;
    __syncthreads();
    interp_items(data, numdata, n, s);
    if (threadIdx.x == 0) {
        int k = 0;
        for (int ii = 0; ii < nh; ii++) {
            double sum = 0.0;
            for (int c = 0; c < s.cnt[ii]; c++, k++) sum += powerf2(s.amp[k]);
            s.locpow[ii] = (float) (sum / (double) PL_LOCPOW);
        }
    }
    __syncthreads();
}

// Minus the summed normalised power of the harmonics at (r, zs * ZSCALE)
// (power_call_rz_harmonics_gsl, src/maximize_rz.c:42-62); all threads.
__device__ double eval_harmonics(const float2 *data, long long numdata, int nh, int kernhw, double r,
                                 double zs, PolishSmem &s)
{
    // P warps per harmonic (all warps busy for few harmonics)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int P = nh >= PL_WARPS ? 1 : PL_WARPS / nh;
    for (int w = warp; w < nh * P; w += PL_WARPS) {
        const int ii = w / P, n = ii + 1;
        const double2 v = warp_sum(rz_interp_part(data, numdata, r * n, zs * PL_ZSCALE * n, kernhw,
                                                  w - ii * P, P, lane));
        if (lane == 0) s.part[w] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double total = 0.0;
        for (int ii = 0; ii < nh; ii++) {
            double ar = 0.0, ai = 0.0;
            for (int q = 0; q < P; q++) {
                ar += s.part[ii * P + q].x;
                ai += s.part[ii * P + q].y;
            }
            const float2 a = make_float2((float) ar, (float) ai);
            s.term[ii] = s.raw ? powerf2(a) : powerf2(a) / (double) s.locpow[ii];
            total += s.term[ii];
        }
        // power_call_rz (src/maximize_rz.c:10-23) for one raw power
        s.val = s.raw ? -total : (isfinite(total) ? -total : 0.0);
    }
    __syncthreads();
    const double v = s.val;
    __syncthreads();
    return v;
}

// Nelder-Mead over (r, zs), the oracle's orc_nm_minimize step for step.
__device__ double nm_minimize(const float2 *data, long long numdata, int nh, int kernhw, double *x,
                              double step, double tol, PolishSmem &s)
{
    double v[3][2], fv[3], xt[2], xt2[2];
    for (int i = 0; i < 3; i++) {
        v[i][0] = x[0];
        v[i][1] = x[1];
        if (i > 0) v[i][i - 1] += step;
        fv[i] = eval_harmonics(data, numdata, nh, kernhw, v[i][0], v[i][1], s);
    }
    for (int iter = 0; iter < 5000; iter++) {
        int hi = 0, lo = 0;
        for (int i = 1; i < 3; i++) {
            if (fv[i] > fv[hi]) hi = i;
            if (fv[i] < fv[lo]) lo = i;
        }
        int shi = (hi == 0) ? 1 : 0;
        for (int i = 0; i < 3; i++)
            if (i != hi && fv[i] > fv[shi]) shi = i;
        double c[2] = {0.0, 0.0};
        for (int i = 0; i < 3; i++)
            if (i != hi) {
                c[0] += v[i][0];
                c[1] += v[i][1];
            }
        c[0] /= 2;
        c[1] /= 2;
        // x(t) = (1 - t) c + t x_worst
        xt[0] = 2.0 * c[0] - v[hi][0];
        xt[1] = 2.0 * c[1] - v[hi][1];
        const double fr = eval_harmonics(data, numdata, nh, kernhw, xt[0], xt[1], s);
        if (fr < fv[lo]) {
            xt2[0] = 3.0 * c[0] - 2.0 * v[hi][0];
            xt2[1] = 3.0 * c[1] - 2.0 * v[hi][1];
            const double fe = eval_harmonics(data, numdata, nh, kernhw, xt2[0], xt2[1], s);
            if (fe < fv[lo]) {
                v[hi][0] = xt2[0];
                v[hi][1] = xt2[1];
                fv[hi] = fe;
            } else {
                v[hi][0] = xt[0];
                v[hi][1] = xt[1];
                fv[hi] = fr;
            }
        } else if (fr > fv[shi]) {
            if (fr <= fv[hi]) {
                v[hi][0] = xt[0];
                v[hi][1] = xt[1];
                fv[hi] = fr;
            }
            xt2[0] = 0.5 * c[0] + 0.5 * v[hi][0];
            xt2[1] = 0.5 * c[1] + 0.5 * v[hi][1];
            const double fc = eval_harmonics(data, numdata, nh, kernhw, xt2[0], xt2[1], s);
            if (fc <= fv[hi]) {
                v[hi][0] = xt2[0];
                v[hi][1] = xt2[1];
                fv[hi] = fc;
            } else {
                for (int i = 0; i < 3; i++) {
                    if (i == lo) continue;
                    v[i][0] = 0.5 * (v[i][0] + v[lo][0]);
                    v[i][1] = 0.5 * (v[i][1] + v[lo][1]);
                    fv[i] = eval_harmonics(data, numdata, nh, kernhw, v[i][0], v[i][1], s);
                }
            }
        } else {
            v[hi][0] = xt[0];
            v[hi][1] = xt[1];
            fv[hi] = fr;
        }
        double m0 = 0.0, m1 = 0.0, s2 = 0.0;
        for (int i = 0; i < 3; i++) {
            m0 += v[i][0] / 3;
            m1 += v[i][1] / 3;
        }
        for (int i = 0; i < 3; i++) {
            s2 += (v[i][0] - m0) * (v[i][0] - m0);
            s2 += (v[i][1] - m1) * (v[i][1] - m1);
        }
        if (sqrt(s2 / 3) < tol) break;
    }
    int lo = 0;
    for (int i = 1; i < 3; i++)
        if (fv[i] < fv[lo]) lo = i;
    x[0] = v[lo][0];
    x[1] = v[lo][1];
    return fv[lo];
}

__global__ void __launch_bounds__(PL_THREADS) k_polish_rz(const float2 *data, long long numdata,
                                                          long long lobin, const PolishIn *in,
                                                          ab_polished *out)
{
    __shared__ PolishSmem s;
    const PolishIn c = in[blockIdx.x];
    ab_polished &o = out[blockIdx.x];
    const int nh = c.mode == 1 ? 1 : (c.numharm < 1 ? 1 : (c.numharm > PL_MAXH ? PL_MAXH : c.numharm));
    if (threadIdx.x == 0) s.raw = c.mode == 1;
    const double rin = c.r - (double) lobin, zin = c.z;
    local_powers(data, numdata, rin, zin, nh, s);
    double x[2] = {rin, zin / PL_ZSCALE};
    int kernhw = z_halfwidth(fabs(zin * nh) + 4.0, false);
    nm_minimize(data, numdata, nh, kernhw, x, 0.4, 1.0e-4, s);
    kernhw = z_halfwidth(fabs(x[1] * nh) + 4.0, true);
    nm_minimize(data, numdata, nh, kernhw, x, 0.01, 1.0e-7, s);
    const double rout = x[0], zout = x[1] * PL_ZSCALE;
    local_powers(data, numdata, rout, zout, nh, s);
    // harmonic powers (HIGHACC kernel of the second stage) and the five
    // derivative points r n - 0.006 .. + 0.006 (get_derivs3d) per harmonic
    if (threadIdx.x == 0) {
        for (int ii = 0; ii < nh; ii++) {
            const int n = ii + 1;
            const double zs = zout / PL_ZSCALE * n;
            s.r[ii] = rout * n;
            s.z[ii] = zs * PL_ZSCALE;
            s.hw[ii] = kernhw;
            const int hwd = z_halfwidth(zout * n, true);
            double f = rout * n - 0.006;
            for (int q = 0; q < 5; q++, f += 0.003) {
                const int k = PL_MAXH + 5 * ii + q;
                s.r[k] = f;
                s.z[k] = zout * n;
                s.hw[k] = hwd;
            }
        }
    }
    __syncthreads();
    // items: [0, nh) powers, [PL_MAXH, PL_MAXH + 5 nh) derivative points
    {
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        for (int it = warp; it < PL_MAXH + 5 * nh; it += PL_WARPS) {
            if (it >= nh && it < PL_MAXH) continue;
            const float2 a = warp_rz_interp(data, numdata, s.r[it], s.z[it], s.hw[it], lane);
            if (lane == 0) s.amp[it] = a;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double pi = 3.14159265358979323846, twopi = 6.28318530717958647692;
        o.numharm = nh;
        for (int ii = 0; ii < nh; ii++) {
            const int n = ii + 1;
            o.hirs[ii] = (rout + (double) lobin) * n;
            o.hizs[ii] = zout * n;
            o.hiws[ii] = 0.0;
            o.pows[ii] = powerf2(s.amp[ii]);
            double pwr[5], phs[5];
            for (int q = 0; q < 5; q++) {
                const float2 a = s.amp[PL_MAXH + 5 * ii + q];
                pwr[q] = powerf2(a);
                const double t = atan2((double) a.y, (double) a.x);
                phs[q] = t > 0.0 ? t : t + twopi;
            }
            for (int q = 0; q < 4; q++)
                if (fabs(phs[q + 1] - phs[q]) > pi) phs[q + 1] -= twopi;
            ab_rderivs &d = o.derivs[ii];
            d.pow = pwr[2];
            d.phs = phs[2];
            d.dpow = (pwr[3] - pwr[1]) / 0.006;
            d.dphs = (phs[3] - phs[1]) / 0.006;
            d.d2pow = (pwr[4] - 2.0 * pwr[2] + pwr[0]) / 0.000036;
            d.d2phs = (phs[4] - 2.0 * phs[2] + phs[0]) / 0.000036;
            d.locpow = (double) s.locpow[ii];
        }
    }
}

}  // namespace

cudaError_t launch_polish(const float2 *data, long long numdata, long long lobin, const PolishIn *in,
                          int n, ab_polished *out, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    k_polish_rz<<<n, PL_THREADS, 0, st>>>(data, numdata, lobin, in, out);
    return cudaGetLastError();
}

}  // namespace ab
