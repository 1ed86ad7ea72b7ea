// ab_polish_rzw.cu -- jerk-search candidate polishing on the device:
// max_rzw_arr_harmonics (src/maximize_rzw.c:81-191) as called by
// optimize_accelcand for numw > 0 (src/accel_utils.c:552-626).
//
// The reference's work per candidate is, per harmonic, 17 x 17 responses
// gen_w_response(0, 8, z, w, 16 hw) (src/responses.c:333-418: a chirp of
// npts samples zero padded to 8 npts and Fourier transformed) correlated with
// the spectrum (corr_rzw_vol, src/rzwinterp.c:3-140), then a sum over
// harmonics and an arg-max, then get_localpower3d / get_derivs3d
// (src/characteristics.c:79-193), each a handful of rzw_interp calls with
// their own responses.  Here every response is a job of k_rzw_jobs (one CTA):
//
//  * the zero-padded transform X[g], g = nb k + s, of a chirp x[t], t < N,
//    is computed phase by phase: with N = M P (P <= 4096) and t = M a + b,
//      X[nb k + s] = sum_b W_N^{k b} W_{nb N}^{s b}
//                      FFT_P( x[M a + b] W_{nb P}^{s a} )[k mod P],
//    one FP64 radix-2 FFT of P points in shared memory per (b, s), the
//    chirp samples of one b kept in shared memory across the nb phases;
//    only the numkern outputs the reference keeps are formed, rounded to
//    float as the reference stores its response;
//  * the job's correlation outputs (the 24 r cells of a volume row, or an
//    rzw_interp point) are FP64 dot products, one warp each.
// k_rzw_sum then forms the summed, locally normalised powers in float in the
// reference's order and picks the first highest cell.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "ab_index.h"
#include "ab_kernels.h"
#include "ab_resp.cuh"

namespace ab {

namespace {

constexpr int RZW_THREADS = 512;
constexpr long long RZW_NMAX = 1LL << RZW_NMAX_LOG2;

// exp(-2 pi i m / RZW_NMAX) from the half-circle table tw[m] (m < NMAX / 2)
__device__ __forceinline__ double2 tw_at(const double2 *tw, long long m)
{
    m &= RZW_NMAX - 1;
    if (m < RZW_NMAX / 2) return tw[m];
    const double2 v = tw[m - RZW_NMAX / 2];
    return make_double2(-v.x, -v.y);
}

__device__ __forceinline__ double2 cmul64(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Forward FP64 FFT of n = 2^log2n points in shared memory (radix 2,
// decimation in time after a bit reversal).  All threads of the CTA call it;
// it ends with a barrier.
__device__ void fft_pow2(double2 *x, int n, int log2n, const double2 *tw)
{
    const long long tstride = RZW_NMAX / n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int j = (int) (__brev((unsigned) i) >> (32 - log2n));
        if (j > i) {
            const double2 a = x[i];
            x[i] = x[j];
            x[j] = a;
        }
    }
    __syncthreads();
    for (int lh = 0; lh < log2n; lh++) {
        const int half = 1 << lh;
        const long long st = (long long) (n >> (lh + 1)) * tstride;
        for (int b = threadIdx.x; b < n / 2; b += blockDim.x) {
            const int k = b & (half - 1);
            const int i0 = ((b >> lh) << (lh + 1)) + k, i1 = i0 + half;
            const double2 w = tw[k * st];
            const double2 u = x[i0], v = cmul64(x[i1], w);
            x[i0] = make_double2(u.x + v.x, u.y + v.y);
            x[i1] = make_double2(u.x - v.x, u.y - v.y);
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(RZW_THREADS) k_rzw_jobs(const RzwJob *jobs, const float2 *data,
                                                          long long numdata, const double2 *tw,
                                                          float2 *resp_all, double2 *acc_all,
                                                          const long long *out_j, float2 *out_amp)
{
    extern __shared__ double2 sm[];
    const RzwJob jb = jobs[blockIdx.x];
    if (jb.mode == 2) {
        if (threadIdx.x == 0) {
            const long long b = jb.beginbin;
            out_amp[jb.out_off] = (b >= 0 && b < numdata) ? data[b] : make_float2(0.f, 0.f);
        }
        return;
    }
    const int nb = jb.nb, numkern = jb.numkern;
    float2 *resp = resp_all + jb.resp_off;
    if (jb.mode == 0) {
        for (int c = threadIdx.x; c < numkern; c += blockDim.x) {
            const double2 v = z_resp_point(jb.roffset, nb, jb.z, numkern, c);
            resp[c] = make_float2((float) v.x, (float) v.y);
        }
    } else {
        const int N = jb.npts, P = N < RZW_PMAX ? N : RZW_PMAX, M = N / P;
        const int logP = 31 - __clz(P);
        double2 *y = sm;                                        // [P]
        double *xb = reinterpret_cast<double *>(sm + P);        // [P]
        const double dt = 1.0 / (double) N, amp = 2.0 * dt;
        const int fbar = N / 4;
        const double f = ((double) fbar + jb.roffset) - 0.5 * jb.z + jb.w / 12.0;
        const double fd = (jb.z - 0.5 * jb.w) / 2.0, fdd = jb.w / 6.0;
        // first kept output g0 = fbar nb - numkern / 2, a multiple of nb
        const long long kbase = (long long) fbar - numkern / (2 * nb);
        const long long sP = RZW_NMAX / ((long long) nb * P), sN = RZW_NMAX / N;
        double2 *acc = (M > 1) ? acc_all + jb.acc_off : nullptr;
        for (int b = 0; b < M; b++) {
            for (int q = threadIdx.x; q < P; q += blockDim.x) {
                const double t = (double) (q * M + b) * dt;
                xb[q] = amp * cospi(2.0 * (t * (t * (t * fdd + fd) + f)));
            }
            for (int s = 0; s < nb; s++) {
                // same q per thread as above: xb[q] is this thread's own write
                for (int q = threadIdx.x; q < P; q += blockDim.x) {
                    const double2 w = tw_at(tw, (long long) s * q * sP);
                    y[q] = make_double2(xb[q] * w.x, xb[q] * w.y);
                }
                __syncthreads();
                fft_pow2(y, P, logP, tw);
                double2 wsb = make_double2(1.0, 0.0);
                if (M > 1 && s * b != 0) {
                    double sn, cs;
                    sincospi(-2.0 * (double) (s * b) / ((double) nb * (double) N), &sn, &cs);
                    wsb = make_double2(cs, sn);
                }
                // outputs c = s, s + nb, ...: g = g0 + c = nb (kbase + (c - s) / nb) + s
                for (int c = s + nb * (int) threadIdx.x; c < numkern; c += nb * (int) blockDim.x) {
                    const long long k = kbase + (c - s) / nb;
                    double2 v = y[k & (P - 1)];
                    if (M == 1) {
                        resp[c] = make_float2((float) v.x, (float) v.y);
                    } else {
                        v = cmul64(v, cmul64(tw_at(tw, ((k * b) & (N - 1)) * sN), wsb));
                        if (b > 0) v = make_double2(acc[c].x + v.x, acc[c].y + v.y);
                        if (b == M - 1) resp[c] = make_float2((float) v.x, (float) v.y);
                        else acc[c] = v;
                    }
                }
                __syncthreads();            // y and xb are rewritten next
            }
        }
    }
    __syncthreads();                        // the response is visible to the whole CTA
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (int o = warp; o < jb.nout; o += nwarp) {
        const long long j = out_j[jb.j_off + o];
        const long long i0 = j >= 0 ? (j + nb - 1) / nb : -((-j) / nb);
        const long long i1 = (numkern - 1 + j) / nb;
        double ar = 0.0, ai = 0.0;
        for (long long i = i0 + lane; i <= i1; i += 32) {
            const long long bi = jb.beginbin + i;
            if (bi < 0 || bi >= numdata) continue;
            const float2 d = data[bi], p = resp[nb * i - j];
            ar += (double) d.x * p.x + (double) d.y * p.y;
            ai += (double) d.y * p.x - (double) d.x * p.y;
        }
#pragma unroll
        for (int m = 16; m > 0; m >>= 1) {
            ar += __shfl_xor_sync(0xffffffffu, ar, m);
            ai += __shfl_xor_sync(0xffffffffu, ai, m);
        }
        if (lane == 0) out_amp[jb.out_off + o] = make_float2((float) ar, (float) ai);
    }
}

// One CTA per candidate.  Local powers: get_localpower3d's double sum of
// |amp|^2 over its points in order, / NUMLOCPOWAVG, to float
// (src/characteristics.c:79-127); summed powers: float |vol|^2 / locpow
// added from the highest harmonic down (src/maximize_rzw.c:134-140), every
// operation rounded on its own as the reference's scalar code rounds it.
__global__ void __launch_bounds__(256) k_rzw_sum(const float2 *amp, const int *numharm,
                                                 const int *vol_off, const int *lp_off,
                                                 const int *lp_n, int ncell, int *best,
                                                 float *bestval)
{
    __shared__ float s_locpow[AB_POLISH_MAX_HARM];
    __shared__ float s_p[256];
    __shared__ int s_i[256];
    const int c = blockIdx.x, nh = numharm[c];
    if ((int) threadIdx.x < nh) {
        const int h = threadIdx.x;
        const int n = lp_n[c * AB_POLISH_MAX_HARM + h];
        const float2 *a = amp + lp_off[c * AB_POLISH_MAX_HARM + h];
        double sum = 0.0;
        for (int m = 0; m < n; m++)
            sum = __dadd_rn(sum, __dadd_rn(__dmul_rn((double) a[m].x, (double) a[m].x),
                                           __dmul_rn((double) a[m].y, (double) a[m].y)));
        // n < 0: raw powers (max_rzw_arr); x / 1 is x
        s_locpow[h] = n < 0 ? 1.0f : (float) (sum / 20.0);
    }
    __syncthreads();
    float bp = 0.0f;
    int bi = ncell;                         // none above zero yet
    const float2 *vol = amp + vol_off[c];
    for (int cell = threadIdx.x; cell < ncell; cell += blockDim.x) {
        float ps = 0.0f;
        for (int h = 0; h < nh; h++) {
            const float2 v = vol[h * ncell + cell];
            const float p = __fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y));
            ps = __fadd_rn(ps, __fdiv_rn(p, s_locpow[h]));
        }
        if (ps > bp) {
            bp = ps;
            bi = cell;
        }
    }
    s_p[threadIdx.x] = bp;
    s_i[threadIdx.x] = bi;
    __syncthreads();
    for (int m = 128; m > 0; m >>= 1) {
        if ((int) threadIdx.x < m) {
            const float po = s_p[threadIdx.x + m];
            const int io = s_i[threadIdx.x + m];
            if (po > s_p[threadIdx.x] || (po == s_p[threadIdx.x] && io < s_i[threadIdx.x])) {
                s_p[threadIdx.x] = po;
                s_i[threadIdx.x] = io;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        best[c] = s_i[0] == ncell ? 0 : s_i[0];
        if (bestval) bestval[c] = s_i[0] == ncell ? 0.0f : s_p[0];
    }
}

}  // namespace

cudaError_t launch_rzw_jobs(const RzwJob *jobs, int njobs, const float2 *data, long long numdata,
                            const double2 *tw, float2 *resp, double2 *acc, const long long *out_j,
                            float2 *out_amp, cudaStream_t st)
{
    if (njobs <= 0) return cudaSuccess;
    const size_t smem = (size_t) RZW_PMAX * (sizeof(double2) + sizeof(double));
    cudaError_t e = cudaFuncSetAttribute(k_rzw_jobs, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int) smem);
    if (e != cudaSuccess) return e;
    k_rzw_jobs<<<njobs, RZW_THREADS, smem, st>>>(jobs, data, numdata, tw, resp, acc, out_j, out_amp);
    return cudaGetLastError();
}

cudaError_t launch_rzw_sum(const float2 *amp, const int *numharm, const int *vol_off,
                           const int *lp_off, const int *lp_n, int ncell, int ncand, int *best,
                           float *bestval, cudaStream_t st)
{
    if (ncand <= 0) return cudaSuccess;
    k_rzw_sum<<<ncand, 256, 0, st>>>(amp, numharm, vol_off, lp_off, lp_n, ncell, best, bestval);
    return cudaGetLastError();
}

}  // namespace ab

// ---------------------------------------------------------------------------
// Host side: the reference's geometry in FP64, planned into response jobs.
// ---------------------------------------------------------------------------
namespace ab {

namespace {

constexpr double kTwoPi = 6.28318530717958647692528676655900576;
constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr int kInterpFac = 4, kNumWid = 2;              // src/maximize_rzw.c:92-93
constexpr int kRzwNb = kInterpFac * 2;                 // interpfac * ACCEL_RDR
constexpr int kNumR = 3 * kRzwNb, kNumZ = 2 * kNumWid * kInterpFac + 1;
static_assert(kNumZ * kNumZ * kNumR == RZW_VOL, "volume cells");
constexpr double kAccelDZ = 2.0, kAccelDW = 20.0;      // include/accel.h:25,29

// w_resp_halfwidth with LOWACC or HIGHACC (src/responses.c:27-84): HIGHACC
// adds 3 x NUMFINTBINS instead of NUMFINTBINS.
int w_halfwidth(double z, double w, bool highacc)
{
    return ab_resp_halfwidth(z, w) + (highacc ? 2 * AB_NUMFINTBINS : 0);
}

long long next2(long long x)
{
    long long n = 1;
    while (n < x) n <<= 1;
    return n;
}

struct Plan {
    long long numdata = 0;
    std::vector<RzwJob> jobs;
    std::vector<long long> js;              // correlation offsets j of the outputs
    long long namp = 0;                     // amplitudes (outputs) so far
    bool bad = false;
    char msg[200] = {0};

    int outputs() const { return (int) namp; }

    static long long chirp_points(double z, double w, int numkern, int nb)
    {
        // gen_w_response's num_pts_wdat (src/responses.c:381-382)
        return next2(6LL * ab_resp_halfwidth(z, w) + 200 + numkern / nb);
    }
    void check_chirp(const RzwJob &jb)
    {
        if (jb.npts > RZW_NMAX || (jb.npts / 4) * jb.nb < jb.numkern / 2) {
            bad = true;
            snprintf(msg, sizeof msg, "response (z %.1f, w %.1f) needs %d chirp samples, "
                     "above %lld", jb.z, jb.w, jb.npts, RZW_NMAX);
        }
    }

    // A new job (mode 0 / 1) with its first output.
    void open(int mode, double roffset, double z, double w, int nb, int hw, long long beginbin,
              long long j)
    {
        RzwJob jb{};
        jb.mode = mode;
        jb.roffset = roffset;
        jb.z = z;
        jb.w = w;
        jb.nb = nb;
        jb.numkern = 2 * nb * hw;
        jb.beginbin = beginbin;
        jb.out_off = outputs();
        jb.j_off = (int) js.size();
        jb.nout = 0;
        if (mode == 1) {
            const long long npts = chirp_points(z, w, jb.numkern, nb);
            jb.npts = (int) std::min<long long>(npts, 1LL << 30);
            check_chirp(jb);
        }
        jobs.push_back(jb);
        add_output(j);
    }
    // A job with another response (mode, z, w) over the same data window and
    // the same outputs as job `like` (the cells of one volume row).
    void open_like(int like, int mode, double z, double w)
    {
        RzwJob jb = jobs[(size_t) like];
        jb.mode = mode;
        jb.z = z;
        jb.w = w;
        jb.npts = 0;
        if (mode == 1) {
            jb.npts = (int) std::min<long long>(chirp_points(z, w, jb.numkern, jb.nb), 1LL << 30);
            check_chirp(jb);
        }
        jb.out_off = outputs();
        namp += jb.nout;
        jobs.push_back(jb);
    }
    void add_output(long long j)
    {
        RzwJob &jb = jobs.back();
        if (j <= -jb.numkern && jb.mode != 2) {
            bad = true;
            snprintf(msg, sizeof msg, "correlation offset %lld outside a %d-point response", j,
                     jb.numkern);
        }
        if (jb.j_off + jb.nout != (int) js.size() || jb.out_off + jb.nout != namp) {
            bad = true;                     // a shared list can not grow
            snprintf(msg, sizeof msg, "jerk polishing plan: output appended to a shared list");
        }
        js.push_back(j);
        jb.nout++;
        namp++;
    }
    void copy_bin(long long bin)
    {
        RzwJob jb{};
        jb.mode = 2;
        jb.beginbin = bin;
        jb.out_off = outputs();
        jb.j_off = (int) js.size();
        jb.nout = 1;
        jobs.push_back(jb);
        js.push_back(0);
        namp++;
    }

    // rzw_interp at r with kern_half_width hw (src/rzwinterp.c:145-228, and
    // rz_interp, src/rzinterp.c:144-232, when |w| < 1e-4).  Appends one
    // output; consecutive points that share the response (same fraction)
    // join the last job when allow_join.  Returns the output index, or -1
    // where the reference returns 0 (r outside the spectrum).
    int point(double r, double z, double w, int hw, bool allow_join)
    {
        if (r > numdata - 1.0 || r < 0.0) return -1;
        double dint;
        const double frac = modf(r, &dint);
        const long long intfreq = (long long) dint;
        const bool usew = fabs(w) >= 1E-4;
        if (!usew && fabs(z) < 1E-4) {
            if (frac < 1E-5) {
                copy_bin(intfreq);
                return outputs() - 1;
            }
            if ((1.0 - frac) < 1E-5) {
                copy_bin(intfreq + 1);
                return outputs() - 1;
            }
        }
        const int mode = usew ? 1 : 0;
        if (allow_join && !jobs.empty()) {
            RzwJob &last = jobs.back();
            if (last.mode == mode && last.nb == 1 && last.roffset == frac && last.z == z &&
                last.w == w && last.numkern == 2 * hw) {
                add_output(intfreq - (last.beginbin + hw));
                return outputs() - 1;
            }
        }
        open(mode, frac, z, w, 1, hw, intfreq - hw, 0);
        return outputs() - 1;
    }

    // get_localpower3d's points (src/characteristics.c:79-127), outputs
    // contiguous from the returned index; *count of them.
    int localpower(double r, double z, double w, int *count)
    {
        const int first = outputs();
        const int binsperside = 20 / 2, hw = w_halfwidth(z, w, false);
        double lo1 = r - 5 - binsperside, hi1 = lo1 + binsperside;
        double lo2 = r + 5, hi2 = lo2 + binsperside;
        double *bd[4] = {&lo1, &lo2, &hi1, &hi2};
        for (double *p : bd) {
            if (*p < 0.0) *p = 0.0;
            if (*p > numdata) *p = (double) numdata;
        }
        bool join = false;
        for (double f = lo1; f < hi1; f += 1.0) join = point(f, z, w, hw, join) >= 0;
        join = false;
        for (double f = lo2; f < hi2; f += 1.0) join = point(f, z, w, hw, join) >= 0;
        *count = outputs() - first;
        return first;
    }
};

// One candidate's search state between the stages.
struct CandState {
    int nh;
    double rin, zin, win;
    long long hhlobin;
    double rout, zout, wout;
    int lp_off[AB_POLISH_MAX_HARM], lp_n[AB_POLISH_MAX_HARM];
    int d_idx[AB_POLISH_MAX_HARM][5];
};

struct DevMem {
    void *p = nullptr;
    size_t n = 0;
    ~DevMem() { if (p) cudaFree(p); }
    cudaError_t ensure(size_t bytes)
    {
        if (bytes <= n) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc(&p, bytes ? bytes : 1);
        if (e == cudaSuccess) n = bytes;
        return e;
    }
};

// Runs the jobs of plan in chunks whose responses fit budget bytes; the
// outputs land in out_amp (plan.outputs() entries).
cudaError_t run_plan(Plan &plan, const float2 *data, const double2 *tw, size_t budget, DevMem &djobs,
                     DevMem &dresp, DevMem &dacc, DevMem &dj, DevMem &damp, cudaStream_t st,
                     long long *launches)
{
    cudaError_t e = dj.ensure(sizeof(long long) * plan.js.size());
    if (e == cudaSuccess) e = damp.ensure(sizeof(float2) * (size_t) plan.namp);
    if (e == cudaSuccess && !plan.js.empty())
        e = cudaMemcpyAsync(dj.p, plan.js.data(), sizeof(long long) * plan.js.size(),
                            cudaMemcpyHostToDevice, st);
    size_t i = 0;
    while (e == cudaSuccess && i < plan.jobs.size()) {
        const size_t j0 = i;
        long long roff = 0, aoff = 0;
        while (i < plan.jobs.size()) {
            RzwJob &jb = plan.jobs[i];
            const long long nr = jb.mode == 2 ? 0 : jb.numkern;
            const long long na = (jb.mode == 1 && jb.npts > RZW_PMAX) ? jb.numkern : 0;
            if (i > j0 && (size_t) ((roff + nr) * 8 + (aoff + na) * 16) > budget) break;
            jb.resp_off = roff;
            jb.acc_off = aoff;
            roff += nr;
            aoff += na;
            i++;
        }
        e = djobs.ensure(sizeof(RzwJob) * (i - j0));
        if (e == cudaSuccess) e = dresp.ensure(sizeof(float2) * (size_t) roff);
        if (e == cudaSuccess) e = dacc.ensure(sizeof(double2) * (size_t) aoff);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(djobs.p, plan.jobs.data() + j0, sizeof(RzwJob) * (i - j0),
                                cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = launch_rzw_jobs((const RzwJob *) djobs.p, (int) (i - j0), data, plan.numdata, tw,
                                (float2 *) dresp.p, (double2 *) dacc.p, (const long long *) dj.p,
                                (float2 *) damp.p, st);
        if (e == cudaSuccess) ++*launches;
    }
    return e;
}

double radian_phase(double re, double im)      // RADIAN_PHASE, include/presto.h:88
{
    const double t = atan2(im, re);
    return t > 0.0 ? t : t + kTwoPi;
}

}  // namespace

int rzw_optimize(const float2 *data, long long numdata, long long lobin, const ab_cand *cands,
                 long long n, ab_polished *out, const double2 *tw, size_t budget, cudaStream_t st,
                 char *err, size_t errlen, long long *launches)
{
    // every output of the plan is indexed by int: bound the call's volume
    long long nharm = 0;
    for (long long c = 0; c < n; c++) nharm += cands[c].numharm;
    if (nharm * (long long) (RZW_VOL + 64) > (1LL << 27)) {
        snprintf(err, errlen, "%lld harmonics to polish in one call: at most %lld", nharm,
                 (1LL << 27) / (RZW_VOL + 64));
        return AB_ERR_ARG;
    }
    std::vector<CandState> cs((size_t) n);
    Plan pv;
    pv.numdata = numdata;
    std::vector<int> nh((size_t) n), vol_off((size_t) n);
    std::vector<int> lp_off((size_t) n * AB_POLISH_MAX_HARM, 0), lp_n((size_t) n * AB_POLISH_MAX_HARM, 0);
    // stage 1: per harmonic, from the highest, its local power and volume
    // (src/maximize_rzw.c:107-141)
    for (long long c = 0; c < n; c++) {
        CandState &s = cs[c];
        s.nh = cands[c].numharm;
        s.rin = cands[c].r - (double) lobin;
        s.zin = cands[c].z;
        s.win = cands[c].w;
        nh[c] = s.nh;
        for (int hind = 0; hind < s.nh; hind++) {
            const int hn = s.nh - hind;
            int cnt = 0;
            lp_off[c * AB_POLISH_MAX_HARM + hind] =
                pv.localpower(s.rin * hn, s.zin * hn, s.win * hn, &cnt);
            lp_n[c * AB_POLISH_MAX_HARM + hind] = cnt;
        }
        vol_off[c] = pv.outputs();
        for (int hind = 0; hind < s.nh; hind++) {
            const int hn = s.nh - hind;
            const double rh = s.rin * hn, zh = s.zin * hn, wh = s.win * hn;
            const double hfrac = hn / (double) s.nh;
            double rh_int;
            modf(rh, &rh_int);
            const long long lobin_h = (long long) rh_int - 1;
            if (hind == 0) s.hhlobin = lobin_h;
            long long rind[kNumR];
            const double dr = 1.0 / (double) kRzwNb;
            for (int kk = 0; kk < kNumR; kk++)
                rind[kk] = (long long) round(((s.hhlobin + kk * dr) * hfrac - lobin_h) * kRzwNb);
            // corr_rzw_vol's grid and kernel width (src/rzwinterp.c:37-60)
            const double zlo = zh - kNumWid * hfrac * kAccelDZ, zhi = zh + kNumWid * hfrac * kAccelDZ;
            const double wlo = wh - kNumWid * hfrac * kAccelDW, whi = wh + kNumWid * hfrac * kAccelDW;
            const double dz = (zhi - zlo) / (kNumZ - 1), dw = (whi - wlo) / (kNumZ - 1);
            const double maxz = (fabs(zlo) < fabs(zhi)) ? zhi : zlo;
            const double maxw = (fabs(wlo) < fabs(whi)) ? whi : wlo;
            const int hw = w_halfwidth(maxz, maxw, false);
            // every cell of the volume reads the same 24 output offsets
            int first = -1;
            for (int ii = 0; ii < kNumZ; ii++)
                for (int jj = 0; jj < kNumZ; jj++) {
                    const double z = zlo + jj * dz, w = wlo + ii * dw;
                    const int mode = fabs(w) < 1E-4 ? 0 : 1;
                    if (first >= 0) {
                        pv.open_like(first, mode, z, w);
                        continue;
                    }
                    pv.open(mode, 0.0, z, w, kRzwNb, hw, lobin_h - hw, rind[0]);
                    for (int kk = 1; kk < kNumR; kk++) pv.add_output(rind[kk]);
                    first = (int) pv.jobs.size() - 1;
                }
        }
    }
    if (pv.bad) {
        snprintf(err, errlen, "%s", pv.msg);
        return AB_ERR_ARG;
    }
    DevMem djobs, dresp, dacc, dj, damp, dsmall;
    cudaError_t e = run_plan(pv, data, tw, budget, djobs, dresp, dacc, dj, damp, st, launches);
    // stage 2: summed powers and the best cell (src/maximize_rzw.c:143-174)
    const size_t small = sizeof(int) * ((size_t) n * (3 + 2 * AB_POLISH_MAX_HARM));
    if (e == cudaSuccess) e = dsmall.ensure(small);
    std::vector<int> best((size_t) n, 0);
    if (e == cudaSuccess) {
        int *d = (int *) dsmall.p;
        int *d_nh = d, *d_vol = d + n, *d_lpo = d + 2 * n, *d_lpn = d_lpo + n * AB_POLISH_MAX_HARM;
        int *d_best = d_lpn + n * AB_POLISH_MAX_HARM;
        e = cudaMemcpyAsync(d_nh, nh.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_vol, vol_off.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_lpo, lp_off.data(), sizeof(int) * lp_off.size(),
                                cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_lpn, lp_n.data(), sizeof(int) * lp_n.size(), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = launch_rzw_sum((const float2 *) damp.p, d_nh, d_vol, d_lpo, d_lpn, RZW_VOL, (int) n,
                               d_best, nullptr, st);
        if (e == cudaSuccess) ++*launches;
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(best.data(), d_best, sizeof(int) * n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (e != cudaSuccess) {
        snprintf(err, errlen, "jerk polishing (volumes): %s", cudaGetErrorString(e));
        return AB_ERR_CUDA;
    }
    // stage 3: each harmonic's local power and derivatives at the optimum
    // (src/maximize_rzw.c:167-183; get_derivs3d, src/characteristics.c:141-193)
    Plan pd;
    pd.numdata = numdata;
    const double h = 0.003, twoh = 0.006, twohsqrd = 0.000036;
    for (long long c = 0; c < n; c++) {
        CandState &s = cs[c];
        const int cell = best[c], wind = cell / (kNumZ * kNumR), zind = (cell / kNumR) % kNumZ;
        const int rbest = cell % kNumR;
        const double nhd = s.nh, dr = 1.0 / (double) kRzwNb;
        s.rout = (s.hhlobin + rbest * dr) / nhd;
        s.zout = ((s.zin * nhd) - kNumWid * 2 + zind * 2 / (double) kInterpFac) / nhd;
        s.wout = ((s.win * nhd) - kNumWid * 20 + wind * 20 / (double) kInterpFac) / nhd;
        for (int ii = 0; ii < s.nh; ii++) {
            const int hh = ii + 1;
            const double rr = s.rout * hh, zz = s.zout * hh, ww = s.wout * hh;
            s.lp_off[ii] = pd.localpower(rr, zz, ww, &s.lp_n[ii]);
            const int hw = w_halfwidth(zz, ww, true);
            double f = rr - twoh;
            for (int q = 0; q < 5; q++, f += h) s.d_idx[ii][q] = pd.point(f, zz, ww, hw, false);
        }
    }
    if (pd.bad) {
        snprintf(err, errlen, "%s", pd.msg);
        return AB_ERR_ARG;
    }
    e = run_plan(pd, data, tw, budget, djobs, dresp, dacc, dj, damp, st, launches);
    std::vector<float2> amp((size_t) pd.namp);
    if (e == cudaSuccess && !amp.empty())
        e = cudaMemcpyAsync(amp.data(), damp.p, sizeof(float2) * amp.size(), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        snprintf(err, errlen, "jerk polishing (derivatives): %s", cudaGetErrorString(e));
        return AB_ERR_CUDA;
    }
    for (long long c = 0; c < n; c++) {
        const CandState &s = cs[c];
        ab_polished &o = out[c];
        memset(&o, 0, sizeof o);
        o.numharm = s.nh;
        for (int ii = 0; ii < s.nh; ii++) {
            double sum = 0.0;
            for (int m = 0; m < s.lp_n[ii]; m++) {
                const float2 a = amp[s.lp_off[ii] + m];
                sum += (double) a.x * a.x + (double) a.y * a.y;
            }
            const float locpow = (float) (sum / 20.0);
            double pwr[5], phs[5];
            for (int q = 0; q < 5; q++) {
                const int idx = s.d_idx[ii][q];
                const float2 a = idx >= 0 ? amp[idx] : make_float2(0.f, 0.f);
                pwr[q] = (double) a.x * a.x + (double) a.y * a.y;
                phs[q] = radian_phase(a.x, a.y);
            }
            for (int q = 0; q < 4; q++)
                if (fabs(phs[q + 1] - phs[q]) > kPi) phs[q + 1] -= kTwoPi;
            ab_rderivs &d = o.derivs[ii];
            d.pow = pwr[2];
            d.phs = phs[2];
            d.dpow = (pwr[3] - pwr[1]) / twoh;
            d.dphs = (phs[3] - phs[1]) / twoh;
            d.d2pow = (pwr[4] - 2.0 * pwr[2] + pwr[0]) / twohsqrd;
            d.d2phs = (phs[4] - 2.0 * phs[2] + phs[0]) / twohsqrd;
            d.locpow = locpow;
            o.pows[ii] = d.pow;
            o.hirs[ii] = (s.rout + (double) lobin) * (ii + 1);
            o.hizs[ii] = s.zout * (ii + 1);
            o.hiws[ii] = s.wout * (ii + 1);
        }
    }
    return AB_OK;
}

}  // namespace ab

namespace ab {

// -noharmpolish on a jerk search: max_rzw_arr (src/maximize_rzw.c:3-52) for
// each harmonic of each candidate on its own, at (r h - lobin, z h, w h):
// a 9 x 9 x 24 volume (z +- ACCEL_DZ, w +- ACCEL_DW, r from (int) r - 1 in
// 1/8 bins) of raw powers, its first highest cell, and get_derivs3d there
// with the local power taken at the starting point
// (src/accel_utils.c:585-597).
int rzw_optimize_each(const float2 *data, long long numdata, long long lobin, const ab_cand *cands,
                      long long n, ab_polished *out, const double2 *tw, size_t budget,
                      cudaStream_t st, char *err, size_t errlen, long long *launches)
{
    constexpr int numz = 2 * kInterpFac + 1, ncell = numz * numz * kNumR;
    struct Entry {
        long long k;
        int ii;
        double rin, zin, win;
        long long startbin;
        int lp_off, lp_n, d_idx[5];
    };
    std::vector<Entry> es;
    for (long long k = 0; k < n; k++)
        for (int ii = 0; ii < cands[k].numharm; ii++) {
            Entry e{};
            e.k = k;
            e.ii = ii;
            e.rin = cands[k].r * (ii + 1) - (double) lobin;
            e.zin = cands[k].z * (ii + 1);
            e.win = cands[k].w * (ii + 1);
            es.push_back(e);
        }
    const long long ne = (long long) es.size();
    if (ne * (long long) (ncell + 64) > (1LL << 27)) {
        snprintf(err, errlen, "%lld harmonics to polish in one call: at most %lld", ne,
                 (1LL << 27) / (ncell + 64));
        return AB_ERR_ARG;
    }
    Plan pv;
    pv.numdata = numdata;
    std::vector<int> nh((size_t) ne, 1), vol_off((size_t) ne);
    std::vector<int> lp_off((size_t) ne * AB_POLISH_MAX_HARM, 0), lp_n((size_t) ne * AB_POLISH_MAX_HARM, -1);
    for (long long q = 0; q < ne; q++) {
        Entry &e = es[q];
        e.startbin = (long long) (int) e.rin - 1;
        const double zlo = e.zin - kAccelDZ, zhi = e.zin + kAccelDZ;
        const double wlo = e.win - kAccelDW, whi = e.win + kAccelDW;
        const double dz = (zhi - zlo) / (numz - 1), dw = (whi - wlo) / (numz - 1);
        const double maxz = (fabs(zlo) < fabs(zhi)) ? zhi : zlo;
        const double maxw = (fabs(wlo) < fabs(whi)) ? whi : wlo;
        const int hw = w_halfwidth(maxz, maxw, false);
        vol_off[q] = pv.outputs();
        int first = -1;
        for (int iw = 0; iw < numz; iw++)
            for (int jz = 0; jz < numz; jz++) {
                const double z = zlo + jz * dz, w = wlo + iw * dw;
                const int mode = fabs(w) < 1E-4 ? 0 : 1;
                if (first >= 0) {
                    pv.open_like(first, mode, z, w);
                    continue;
                }
                pv.open(mode, 0.0, z, w, kRzwNb, hw, e.startbin - hw, 0);
                for (int kk = 1; kk < kNumR; kk++) pv.add_output(kk);
                first = (int) pv.jobs.size() - 1;
            }
    }
    if (pv.bad) {
        snprintf(err, errlen, "%s", pv.msg);
        return AB_ERR_ARG;
    }
    DevMem djobs, dresp, dacc, dj, damp, dsmall;
    cudaError_t e = run_plan(pv, data, tw, budget, djobs, dresp, dacc, dj, damp, st, launches);
    std::vector<int> best((size_t) ne, 0);
    std::vector<float> bestval((size_t) ne, 0.0f);
    const size_t small = sizeof(int) * ((size_t) ne * (4 + 2 * AB_POLISH_MAX_HARM));
    if (e == cudaSuccess) e = dsmall.ensure(small);
    if (e == cudaSuccess) {
        int *d = (int *) dsmall.p;
        int *d_nh = d, *d_vol = d + ne, *d_lpo = d + 2 * ne, *d_lpn = d_lpo + ne * AB_POLISH_MAX_HARM;
        int *d_best = d_lpn + ne * AB_POLISH_MAX_HARM;
        float *d_val = reinterpret_cast<float *>(d_best + ne);
        e = cudaMemcpyAsync(d_nh, nh.data(), sizeof(int) * ne, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_vol, vol_off.data(), sizeof(int) * ne, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_lpo, lp_off.data(), sizeof(int) * lp_off.size(), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_lpn, lp_n.data(), sizeof(int) * lp_n.size(), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = launch_rzw_sum((const float2 *) damp.p, d_nh, d_vol, d_lpo, d_lpn, ncell, (int) ne,
                               d_best, d_val, st);
        if (e == cudaSuccess) ++*launches;
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(best.data(), d_best, sizeof(int) * ne, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(bestval.data(), d_val, sizeof(float) * ne, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (e != cudaSuccess) {
        snprintf(err, errlen, "jerk polishing (volumes): %s", cudaGetErrorString(e));
        return AB_ERR_CUDA;
    }
    // the optimum, the starting point's local power and the derivatives
    Plan pd;
    pd.numdata = numdata;
    const double h = 0.003, twoh = 0.006, twohsqrd = 0.000036;
    std::vector<double> rout((size_t) ne), zout((size_t) ne), wout((size_t) ne);
    for (long long q = 0; q < ne; q++) {
        Entry &en = es[q];
        const int cell = best[q], wind = cell / (numz * kNumR), zind = (cell / kNumR) % numz;
        const int rind = cell % kNumR;
        rout[q] = en.startbin + rind * 0.5 / (double) kInterpFac;
        zout[q] = en.zin - kAccelDZ + zind * 2 / (double) kInterpFac;
        wout[q] = en.win - kAccelDW + wind * 20 / (double) kInterpFac;
        en.lp_off = pd.localpower(en.rin, en.zin, en.win, &en.lp_n);
        const int hw = w_halfwidth(zout[q], wout[q], true);
        double f = rout[q] - twoh;
        for (int p = 0; p < 5; p++, f += h) en.d_idx[p] = pd.point(f, zout[q], wout[q], hw, false);
    }
    if (pd.bad) {
        snprintf(err, errlen, "%s", pd.msg);
        return AB_ERR_ARG;
    }
    e = run_plan(pd, data, tw, budget, djobs, dresp, dacc, dj, damp, st, launches);
    std::vector<float2> amp((size_t) pd.namp);
    if (e == cudaSuccess && !amp.empty())
        e = cudaMemcpyAsync(amp.data(), damp.p, sizeof(float2) * amp.size(), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        snprintf(err, errlen, "jerk polishing (derivatives): %s", cudaGetErrorString(e));
        return AB_ERR_CUDA;
    }
    for (long long k = 0; k < n; k++) {
        memset(&out[k], 0, sizeof out[k]);
        out[k].numharm = cands[k].numharm;
    }
    for (long long q = 0; q < ne; q++) {
        const Entry &en = es[q];
        ab_polished &o = out[en.k];
        double sum = 0.0;
        for (int m = 0; m < en.lp_n; m++) {
            const float2 a = amp[en.lp_off + m];
            sum += (double) a.x * a.x + (double) a.y * a.y;
        }
        const float locpow = (float) (sum / 20.0);
        double pwr[5], phs[5];
        for (int p = 0; p < 5; p++) {
            const int idx = en.d_idx[p];
            const float2 a = idx >= 0 ? amp[idx] : make_float2(0.f, 0.f);
            pwr[p] = (double) a.x * a.x + (double) a.y * a.y;
            phs[p] = radian_phase(a.x, a.y);
        }
        for (int p = 0; p < 4; p++)
            if (fabs(phs[p + 1] - phs[p]) > kPi) phs[p + 1] -= kTwoPi;
        ab_rderivs &d = o.derivs[en.ii];
        d.pow = pwr[2];
        d.phs = phs[2];
        d.dpow = (pwr[3] - pwr[1]) / twoh;
        d.dphs = (phs[3] - phs[1]) / twoh;
        d.d2pow = (pwr[4] - 2.0 * pwr[2] + pwr[0]) / twohsqrd;
        d.d2phs = (phs[4] - 2.0 * phs[2] + phs[0]) / twohsqrd;
        d.locpow = locpow;
        o.pows[en.ii] = bestval[q];
        o.hirs[en.ii] = rout[q] + (double) lobin;
        o.hizs[en.ii] = zout[q];
        o.hiws[en.ii] = wout[q];
    }
    return AB_OK;
}

}  // namespace ab
