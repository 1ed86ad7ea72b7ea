/* polish_oracle.c -- CPU restatement of accelsearch's candidate polishing
 * (optimize_accelcand, src/accel_utils.c:552-626, and what it calls).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the device polishing kernels.
 * Only tests/, the smoke check and bench.py's CPU legs use it.
 *
 * The reference maximises with GSL's Nelder-Mead simplex
 * (gsl_multimin_fminimizer_nmsimplex2, GSL 2.7/2.8, not in the reference
 * tree); orc_nm_minimize below restates that published algorithm (Nelder &
 * Mead 1965 with the GSL manual's size measure, the RMS distance of the
 * vertices from their centre).  Its iterates need not match GSL's step for
 * step; both stop on a size tolerance (1e-7 bins in the second stage), so the
 * optimum agrees to that level.  Parity is pinned on the reference's own
 * optimizer battery (tests/test_maximize_rz.py: injected peaks recovered from
 * perturbed starts, noiseless and noisy, 1-4 harmonics) restated in
 * tests/test_cpu_polish.py. */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "accel_oracle.h"

#define P_NUMFINTBINS  16          /* include/presto.h:107 */
#define P_NUMLOCPOWAVG 20          /* include/presto.h:99 */
#define P_DELTAAVGBINS 5           /* include/presto.h:103 */
#define P_ZSCALE       4.0         /* src/maximize_rz.c:6 */
#define P_PI           3.14159265358979323846264338327950288
#define P_TWOPI        6.28318530717958647692528676655900576
#define P_DBLCORRECT   1e-14

/* z_resp_halfwidth / w_resp_halfwidth with either accuracy
 * (src/responses.c:27-84). */
int orc_z_resp_halfwidth_acc(double z, int highacc)
{
    int m = (int) (0.5 * 1.1 * fabs(z));
    return m + (highacc ? P_NUMFINTBINS * 3 : P_NUMFINTBINS);
}

int orc_w_resp_halfwidth_acc(double z, double w, int highacc)
{
    if (fabs(w) < 1.0e-7) return orc_z_resp_halfwidth_acc(z, highacc);
    double r0 = 0.5 * (w / 6.0 - z), r1 = 0.5 * (w / 6.0 + z);
    double maxdev = fabs(r0) > fabs(r1) ? fabs(r0) : fabs(r1);
    double u_ext = 0.5 - z / w;
    if (u_ext > 0.0 && u_ext < 1.0) {
        double z0 = z - w / 2.0;
        double r_ext = 0.5 * w * u_ext * u_ext + z0 * u_ext + r0;
        maxdev = fabs(r_ext) > maxdev ? fabs(r_ext) : maxdev;
    }
    return (int) (1.1 * maxdev) + (highacc ? P_NUMFINTBINS * 3 : P_NUMFINTBINS);
}

/* rz_interp (src/rzinterp.c:144-232) and rzw_interp (src/rzwinterp.c:140-228):
 * the complex amplitude at fractional r by direct correlation with the
 * response generated at the fractional offset (numbetween 1, 2 hw points),
 * accumulated in float as the reference does. */
void orc_rzw_interp(const orc_fcomplex *data, long numdata, double r, double z, double w,
                    int kern_half_width, orc_fcomplex *ans)
{
    ans->r = 0.0f;
    ans->i = 0.0f;
    if (r > numdata - 1.0 || r < 0.0) return;
    double dint;
    const double frac = modf(r, &dint);
    const long intfreq = (long) dint;
    const int usew = fabs(w) >= 1E-4;
    if (!usew && fabs(z) < 1E-4) {
        if (frac < 1E-5) {
            *ans = data[intfreq];
            return;
        }
        if ((1.0 - frac) < 1E-5) {
            *ans = data[intfreq + 1];
            return;
        }
    }
    const int numkern = 2 * kern_half_width;
    orc_fcomplex *resp = (orc_fcomplex *) malloc(sizeof(orc_fcomplex) * (size_t) numkern);
    if (usew) orc_gen_w_response(frac, 1, z, w, numkern, resp);
    else orc_gen_z_response(frac, 1, z, numkern, resp);
    long lodata = intfreq - kern_half_width, loresp = 0;
    if (lodata < 0) {
        loresp = -lodata;
        lodata = 0;
    }
    const long hidata = intfreq + kern_half_width - 1;
    const long hiresp = (hidata > numdata - 1) ? numkern - hidata + numdata - 1 : numkern;
    const long nsum = hiresp - loresp;
    float ar = 0.0f, ai = 0.0f;
    for (long ii = 0; ii < nsum; ii++) {
        const orc_fcomplex d = data[lodata + ii], p = resp[loresp + ii];
        const double tmpd = d.r, tmpr = p.r;
        const float pii = d.i * p.i;                  /* float product, as in the reference */
        ar = (float) ((double) ar + (tmpd * tmpr + (double) pii));
        ai = (float) ((double) ai + ((double) d.i * tmpr - (double) p.i * tmpd));
    }
    free(resp);
    ans->r = ar;
    ans->i = ai;
}

/* get_localpower3d (src/characteristics.c:79-127): mean power of the
 * interpolated spectrum over NUMLOCPOWAVG bins, half below r - DELTAAVGBINS,
 * half above r + DELTAAVGBINS. */
double orc_get_localpower3d(const orc_fcomplex *data, long numdata, double r, double z, double w)
{
    const int binsperside = P_NUMLOCPOWAVG / 2;
    const int hw = orc_w_resp_halfwidth_acc(z, w, 0);
    double lo1 = r - P_DELTAAVGBINS - binsperside, hi1 = lo1 + binsperside;
    double lo2 = r + P_DELTAAVGBINS, hi2 = lo2 + binsperside;
    double *b[4] = {&lo1, &lo2, &hi1, &hi2};
    for (int k = 0; k < 4; k++) {
        if (*b[k] < 0.0) *b[k] = 0.0;
        if (*b[k] > numdata) *b[k] = (double) numdata;
    }
    double sum = 0.0;
    orc_fcomplex a;
    for (double f = lo1; f < hi1; f += 1.0) {
        orc_rzw_interp(data, numdata, f, z, w, hw, &a);
        sum += (double) a.r * a.r + (double) a.i * a.i;
    }
    for (double f = lo2; f < hi2; f += 1.0) {
        orc_rzw_interp(data, numdata, f, z, w, hw, &a);
        sum += (double) a.r * a.r + (double) a.i * a.i;
    }
    return sum / (double) P_NUMLOCPOWAVG;
}

static double radian_phase(double re, double im)       /* RADIAN_PHASE, include/presto.h:88 */
{
    double t = atan2(im, re);
    return t > 0.0 ? t : t + P_TWOPI;
}

/* get_derivs3d (src/characteristics.c:141-193): power and phase and their
 * first two r-derivatives by central differences (h = 0.003 bins). */
void orc_get_derivs3d(const orc_fcomplex *data, long numdata, double r, double z, double w,
                      double localpower, orc_rderivs *res)
{
    const double h = 0.003, twoh = 0.006, twohsqrd = 0.000036;
    double pwr[5], phs[5], f = r - twoh;
    const int hw = orc_w_resp_halfwidth_acc(z, w, 1);
    orc_fcomplex a;
    for (int ii = 0; ii < 5; ii++, f += h) {
        orc_rzw_interp(data, numdata, f, z, w, hw, &a);
        pwr[ii] = (double) a.r * a.r + (double) a.i * a.i;
        phs[ii] = radian_phase(a.r, a.i);
    }
    for (int ii = 0; ii < 4; ii++)
        if (fabs(phs[ii + 1] - phs[ii]) > P_PI) phs[ii + 1] -= P_TWOPI;
    res->pow = pwr[2];
    res->phs = phs[2];
    res->dpow = (pwr[3] - pwr[1]) / twoh;
    res->dphs = (phs[3] - phs[1]) / twoh;
    res->d2pow = (pwr[4] - 2.0 * pwr[2] + pwr[0]) / twohsqrd;
    res->d2phs = (phs[4] - 2.0 * phs[2] + phs[0]) / twohsqrd;
    res->locpow = localpower;
}

/* calc_props (src/characteristics.c:195-264): Middleditch, Deich & Kulkarni
 * (1993) signal properties.  Returns -1 where the reference exits (power or
 * local power below DBLCORRECT). */
int orc_calc_props(const orc_rderivs *d, double r, double z, double w, orc_fourierprops *o)
{
    if (fabs(d->pow) < P_DBLCORRECT || d->locpow < P_DBLCORRECT) return -1;
    const double tmppow = d->pow / d->locpow, tmpd2pow = d->d2pow / d->locpow;
    o->pur = (float) (sqrt(1.5 * fabs(tmpd2pow) / tmppow) / P_PI);
    if (fabs(tmppow) < P_DBLCORRECT) o->pur = 1.0f;
    o->purerr = (float) (1.0 / (o->pur * sqrt(10.0 * tmppow)));
    o->r = r;
    o->rerr = (float) (3.0 / (P_PI * o->pur * sqrt(6.0 * tmppow)));
    o->z = z;
    o->zerr = (float) (3.0 * sqrt(10.0) / (P_PI * o->pur * o->pur * sqrt(tmppow)));
    o->w = w;
    o->werr = (float) (6.0 * sqrt(105.0) / (P_PI * o->pur * o->pur * o->pur * sqrt(tmppow)));
    o->pow = (float) tmppow;
    o->powerr = (float) sqrt(2.0 * tmppow);
    o->sig = (float) sqrt(2.0 * tmppow - log(P_PI * tmppow));
    o->rawpow = (float) d->pow;
    o->phs = (float) d->phs;
    o->phserr = (float) (1.0 / o->powerr);
    o->cen = (float) (-d->dphs / P_TWOPI);
    o->cenerr = (float) (1.0 / sqrt(24.0 * tmppow));
    o->locpow = (float) d->locpow;
    return 0;
}

/* ---------------------------------------------------------------------- */
/* Nelder-Mead simplex (the algorithm of gsl_multimin_fminimizer_nmsimplex2)
 * in n <= 3 dimensions.  Initial simplex: x and x + step e_k.  Each
 * iteration moves the worst vertex along the line through the centroid c of
 * the others, x(t) = (1 - t) c + t x_worst: reflection t = -1; if that beats
 * the best vertex, expansion t = -2 (kept if it also beats the best vertex);
 * if the reflection is worse than the second-worst vertex, it replaces the
 * worst only if better than it, then contraction t = 1/2 is tried and, failing
 * that, every vertex moves half-way to the best.  Stops when the RMS distance
 * of the vertices from their centre drops below tol or after maxiter
 * iterations.  Returns f at the best vertex, which is left in x. */
typedef double (*orc_nm_fn)(const double *x, void *par);

static double nm_move(orc_nm_fn f, void *par, int n, double v[4][3], int hi, double t,
                      double *out)
{
    double c[3] = {0, 0, 0};
    for (int i = 0; i <= n; i++)
        if (i != hi)
            for (int k = 0; k < n; k++) c[k] += v[i][k];
    for (int k = 0; k < n; k++) {
        c[k] /= n;
        out[k] = (1.0 - t) * c[k] + t * v[hi][k];
    }
    return f(out, par);
}

double orc_nm_minimize(orc_nm_fn f, void *par, int n, double *x, double step, double tol,
                       int maxiter)
{
    double v[4][3], fv[4], xt[3], xt2[3];
    for (int i = 0; i <= n; i++) {
        for (int k = 0; k < n; k++) v[i][k] = x[k];
        if (i > 0) v[i][i - 1] += step;
        fv[i] = f(v[i], par);
    }
    for (int iter = 0; iter < maxiter; iter++) {
        int hi = 0, lo = 0;
        for (int i = 1; i <= n; i++) {
            if (fv[i] > fv[hi]) hi = i;
            if (fv[i] < fv[lo]) lo = i;
        }
        int shi = (hi == 0) ? 1 : 0;
        for (int i = 0; i <= n; i++)
            if (i != hi && fv[i] > fv[shi]) shi = i;
        const double fr = nm_move(f, par, n, v, hi, -1.0, xt);
        if (fr < fv[lo]) {
            const double fe = nm_move(f, par, n, v, hi, -2.0, xt2);
            if (fe < fv[lo]) {
                memcpy(v[hi], xt2, sizeof(double) * n);
                fv[hi] = fe;
            } else {
                memcpy(v[hi], xt, sizeof(double) * n);
                fv[hi] = fr;
            }
        } else if (fr > fv[shi]) {
            if (fr <= fv[hi]) {
                memcpy(v[hi], xt, sizeof(double) * n);
                fv[hi] = fr;
            }
            const double fc = nm_move(f, par, n, v, hi, 0.5, xt2);
            if (fc <= fv[hi]) {
                memcpy(v[hi], xt2, sizeof(double) * n);
                fv[hi] = fc;
            } else {
                for (int i = 0; i <= n; i++) {
                    if (i == lo) continue;
                    for (int k = 0; k < n; k++) v[i][k] = 0.5 * (v[i][k] + v[lo][k]);
                    fv[i] = f(v[i], par);
                }
            }
        } else {
            memcpy(v[hi], xt, sizeof(double) * n);
            fv[hi] = fr;
        }
        double m[3] = {0, 0, 0}, s2 = 0.0;
        for (int i = 0; i <= n; i++)
            for (int k = 0; k < n; k++) m[k] += v[i][k] / (n + 1);
        for (int i = 0; i <= n; i++)
            for (int k = 0; k < n; k++) s2 += (v[i][k] - m[k]) * (v[i][k] - m[k]);
        if (sqrt(s2 / (n + 1)) < tol) break;
    }
    int lo = 0;
    for (int i = 1; i <= n; i++)
        if (fv[i] < fv[lo]) lo = i;
    memcpy(x, v[lo], sizeof(double) * n);
    return fv[lo];
}

/* ---------------------------------------------------------------------- */
/* max_rz_arr / max_rz_arr_harmonics (src/maximize_rz.c:107-228): simplex
 * over (r, z / ZSCALE), first with LOWACC kernels (step 0.4, tol 1e-4), then
 * from that optimum with HIGHACC kernels (step 0.01, tol 1e-7).  As in the
 * reference, the second stage's half-width is taken from the scaled z. */
typedef struct {
    const orc_fcomplex *data;
    long numdata;
    const float *locpows;
    int numharm, kernhw;
} rz_par;

static double rz_power(double r, double zs, const rz_par *p)
{
    orc_fcomplex a;
    orc_rzw_interp(p->data, p->numdata, r, zs * P_ZSCALE, 0.0, p->kernhw, &a);
    return -((double) a.r * a.r + (double) a.i * a.i);
}

static double rz_fn(const double *x, void *par) { return rz_power(x[0], x[1], (const rz_par *) par); }

static double rz_harm_fn(const double *x, void *par)
{
    const rz_par *p = (const rz_par *) par;
    double total = 0.0;
    for (int ii = 0; ii < p->numharm; ii++) {
        const int n = ii + 1;
        orc_fcomplex a;
        orc_rzw_interp(p->data, p->numdata, x[0] * n, x[1] * P_ZSCALE * n, 0.0, p->kernhw, &a);
        total += ((double) a.r * a.r + (double) a.i * a.i) / p->locpows[ii];
    }
    return isfinite(total) ? -total : 0.0;
}

double orc_max_rz_arr(const orc_fcomplex *data, long numdata, double rin, double zin,
                      double *rout, double *zout, orc_rderivs *derivs)
{
    rz_par p = {data, numdata, NULL, 1, 0};
    double x[2] = {rin, zin / P_ZSCALE};
    p.kernhw = orc_z_resp_halfwidth_acc(fabs(zin) + 4.0, 0);
    orc_nm_minimize(rz_fn, &p, 2, x, 0.4, 1.0e-4, 5000);
    p.kernhw = orc_z_resp_halfwidth_acc(fabs(x[1]) + 4.0, 1);
    double fval = orc_nm_minimize(rz_fn, &p, 2, x, 0.01, 1.0e-7, 5000);
    *rout = x[0];
    *zout = x[1] * P_ZSCALE;
    double locpow = orc_get_localpower3d(data, numdata, *rout, *zout, 0.0);
    orc_get_derivs3d(data, numdata, *rout, *zout, 0.0, locpow, derivs);
    return -fval;
}

void orc_max_rz_arr_harmonics(const orc_fcomplex *data, long numdata, int numharm, double rin,
                              double zin, double *rout, double *zout, orc_rderivs *derivs,
                              double *powers)
{
    float locpow[ORC_MAX_HARM];
    for (int ii = 0; ii < numharm; ii++)
        locpow[ii] = (float) orc_get_localpower3d(data, numdata, rin * (ii + 1), zin * (ii + 1), 0.0);
    rz_par p = {data, numdata, locpow, numharm, 0};
    double x[2] = {rin, zin / P_ZSCALE};
    p.kernhw = orc_z_resp_halfwidth_acc(fabs(zin * numharm) + 4.0, 0);
    orc_nm_minimize(rz_harm_fn, &p, 2, x, 0.4, 1.0e-4, 5000);
    p.kernhw = orc_z_resp_halfwidth_acc(fabs(x[1] * numharm) + 4.0, 1);
    orc_nm_minimize(rz_harm_fn, &p, 2, x, 0.01, 1.0e-7, 5000);
    *rout = x[0];
    *zout = x[1] * P_ZSCALE;
    for (int ii = 0; ii < numharm; ii++) {
        const int n = ii + 1;
        locpow[ii] = (float) orc_get_localpower3d(data, numdata, *rout * n, *zout * n, 0.0);
        powers[ii] = -rz_power(*rout * n, *zout / P_ZSCALE * n, &p);
        orc_get_derivs3d(data, numdata, *rout * n, *zout * n, 0.0, locpow[ii], &derivs[ii]);
    }
}

/* optimize_accelcand (src/accel_utils.c:552-626) for acceleration searches
 * (numw = 0) with harmonic polishing, the reference's default
 * (src/accel_utils.c:1489-1494), on a spectrum held in memory: the harmonics'
 * optimised r, z, powers and derivatives. */
int orc_optimize_accelcand(const orc_fcomplex *fft, long long numbins, long long lobin,
                           int numharm, double r, double z, double *pows, double *hirs,
                           double *hizs, orc_rderivs *derivs)
{
    if (numharm < 1 || numharm > ORC_MAX_HARM) return -1;
    double ro, zo;
    orc_max_rz_arr_harmonics(fft, (long) numbins, numharm, r - (double) lobin, z, &ro, &zo, derivs,
                             pows);
    for (int ii = 0; ii < numharm; ii++) {
        hirs[ii] = (ro + (double) lobin) * (ii + 1);
        hizs[ii] = zo * (ii + 1);
    }
    return 0;
}

/* Many candidates at once (OpenMP over candidates): per candidate k,
 * pows/hirs/hizs/derivs hold ORC_MAX_HARM entries from k * ORC_MAX_HARM. */
int orc_optimize_cands(const orc_fcomplex *fft, long long numbins, long long lobin, int ncand,
                       const int *numharm, const double *r, const double *z, double *pows,
                       double *hirs, double *hizs, orc_rderivs *derivs, int nthreads)
{
    int bad = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1) reduction(| : bad)
#endif
    for (int k = 0; k < ncand; k++)
        bad |= orc_optimize_accelcand(fft, numbins, lobin, numharm[k], r[k], z[k],
                                      pows + (size_t) k * ORC_MAX_HARM,
                                      hirs + (size_t) k * ORC_MAX_HARM,
                                      hizs + (size_t) k * ORC_MAX_HARM,
                                      derivs + (size_t) k * ORC_MAX_HARM) != 0;
    (void) nthreads;
    return bad ? -1 : 0;
}

/* ---------------------------------------------------------------------- */
/* Jerk searches (numw > 0).
 *
 * corr_rzw_vol (src/rzwinterp.c:3-140) correlates the data window that
 * starts kern_half_width bins below lobin, spread to numbetween points per
 * bin, with each (z, w) response (numbetween points per bin, numkern =
 * 2 numbetween kern_half_width) through FFTs of fftlen points, and keeps the
 * uncontaminated outputs from chopbins = kern_half_width numbetween on
 * (corr_complex, src/corr_routines.c:5-262; complex_corr_conv,
 * src/correlations.c:3-60; chop_complex_ends).  Output j of that volume is,
 * exactly, the direct sum
 *     vol[j] = sum_i d[beginbin + i] conj(resp[numbetween i - j]),
 *     0 <= numbetween i - j < numkern,  beginbin = lobin - kern_half_width,
 * with d = 0 outside the spectrum: the complex amplitude at r = lobin +
 * j / numbetween.  It is computed here as that sum in FP64.  For j < 0 or
 * beyond the volume's numgoodbins the reference reads outside its result
 * array (src/maximize_rzw.c:137 can form rind < 0 for harmonics just below
 * the highest); the sum above gives the amplitude at that r instead. */
void orc_rzw_vol_point(const orc_fcomplex *data, long numdata, long beginbin, int numbetween,
                       long j, const orc_fcomplex *resp, int numkern, orc_fcomplex *out)
{
    const long i0 = j >= 0 ? (j + numbetween - 1) / numbetween : -((-j) / numbetween);
    double ar = 0.0, ai = 0.0;
    for (long i = i0; numbetween * i - j < numkern; i++) {
        const long b = beginbin + i;
        if (b < 0 || b >= numdata) continue;
        const orc_fcomplex d = data[b], p = resp[numbetween * i - j];
        ar += (double) d.r * p.r + (double) d.i * p.i;
        ai += (double) d.i * p.r - (double) d.r * p.i;
    }
    out->r = (float) ar;
    out->i = (float) ai;
}

#define P_ACCEL_DZ 2               /* include/accel.h:25 */
#define P_ACCEL_DW 20              /* include/accel.h:29 */
#define P_ACCEL_RDR 2              /* include/accel.h:23 */

/* next2_to_n (src/misc_utils.c) */
static long p_next2(long x)
{
    long n = 1;
    while (n < x) n <<= 1;
    return n;
}

/* The (numw x numz x numr) power volume of one harmonic, rind[] selecting
 * the r outputs: vol_pow[(ii numz + jj) numr + kk] = |vol[rind[kk]]|^2 in
 * float, as corr_rzw_vol's volume is read. */
static void rzw_volume_powers(const orc_fcomplex *data, long numdata, int numbetween, long lobin,
                              double zlo, double zhi, int numz, double wlo, double whi, int numw,
                              const long *rind, int numr, float *vol_pow)
{
    const double dz = numz == 1 ? 0.0 : (zhi - zlo) / (numz - 1);
    const double maxz = (fabs(zlo) < fabs(zhi)) ? zhi : zlo;
    const double dw = numw == 1 ? 0.0 : (whi - wlo) / (numw - 1);
    const double maxw = (fabs(wlo) < fabs(whi)) ? whi : wlo;
    const int hw = orc_w_resp_halfwidth_acc(maxz, maxw, 0);
    const int numkern = 2 * numbetween * hw;
    orc_fcomplex *resp = (orc_fcomplex *) malloc(sizeof(orc_fcomplex) * (size_t) numkern);
    for (int ii = 0; ii < numw; ii++)
        for (int jj = 0; jj < numz; jj++) {
            orc_gen_w_response(0.0, numbetween, zlo + jj * dz, wlo + ii * dw, numkern, resp);
            for (int kk = 0; kk < numr; kk++) {
                orc_fcomplex a;
                orc_rzw_vol_point(data, numdata, lobin - hw, numbetween, rind[kk], resp, numkern, &a);
                const float pr = a.r, pi = a.i;
                vol_pow[((size_t) ii * numz + jj) * numr + kk] = pr * pr + pi * pi;
            }
        }
    free(resp);
}

/* max_rzw_arr (src/maximize_rzw.c:3-52): the highest power of the volume
 * oversampled 4x around (rin, zin, win), then derivatives there. */
double orc_max_rzw_arr(const orc_fcomplex *data, long numdata, double rin, double zin, double win,
                       double *rout, double *zout, double *wout, orc_rderivs *derivs)
{
    const float locpow = (float) orc_get_localpower3d(data, numdata, rin, zin, win);
    const int interpfac = 4, startbin = (int) rin - 1;
    const int numbetween = interpfac * P_ACCEL_RDR, numr = 3 * interpfac * P_ACCEL_RDR;
    const int numz = 2 * interpfac + 1, numw = numz;
    long rind[3 * 4 * P_ACCEL_RDR];
    for (int kk = 0; kk < numr; kk++) rind[kk] = kk;
    float *vp = (float *) malloc(sizeof(float) * (size_t) numw * numz * numr);
    rzw_volume_powers(data, numdata, numbetween, startbin, zin - P_ACCEL_DZ, zin + P_ACCEL_DZ, numz,
                      win - P_ACCEL_DW, win + P_ACCEL_DW, numw, rind, numr, vp);
    float maxpow = 0.0f;
    int wind = 0, zind = 0, rbest = 0;
    for (int ii = 0; ii < numw; ii++)
        for (int jj = 0; jj < numz; jj++)
            for (int kk = 0; kk < numr; kk++) {
                const float p = vp[((size_t) ii * numz + jj) * numr + kk];
                if (p > maxpow) {
                    maxpow = p;
                    wind = ii;
                    zind = jj;
                    rbest = kk;
                }
            }
    free(vp);
    *rout = startbin + rbest * 0.5 / (double) interpfac;
    *zout = zin - P_ACCEL_DZ + zind * P_ACCEL_DZ / (double) interpfac;
    *wout = win - P_ACCEL_DW + wind * P_ACCEL_DW / (double) interpfac;
    orc_get_derivs3d(data, numdata, *rout, *zout, *wout, locpow, derivs);
    return maxpow;
}

/* max_rzw_arr_harmonics (src/maximize_rzw.c:81-191): per harmonic, from the
 * highest, the volume over z and w in exact harmonic ratios (2 peak widths
 * either side, 4x oversampled) and r on the highest harmonic's grid of 1/8
 * bin, powers divided by the harmonic's local power and summed in float;
 * the best cell gives (r, z, w) and each harmonic's derivatives there. */
void orc_max_rzw_arr_harmonics(const orc_fcomplex *data, long numdata, int numharm, double rin,
                               double zin, double win, double *rout, double *zout, double *wout,
                               orc_rderivs *derivs, double *powers)
{
    const int interpfac = 4, numwid = 2;
    const int numbetween = interpfac * P_ACCEL_RDR, numr = 3 * numbetween;
    const int numz = 2 * numwid * interpfac + 1, numw = numz;
    const double dr = 1.0 / (double) numbetween;
    const size_t ncell = (size_t) numw * numz * numr;
    float *powsum = (float *) calloc(ncell, sizeof(float));
    float *vp = (float *) malloc(sizeof(float) * ncell);
    long hhlobin = 0, rind[3 * 4 * P_ACCEL_RDR];
    for (int hind = 0; hind < numharm; hind++) {
        const int n = numharm - hind;
        const double rh = rin * n, zh = zin * n, wh = win * n;
        const double hfrac = n / (double) numharm;
        const float locpow = (float) orc_get_localpower3d(data, numdata, rh, zh, wh);
        double rh_int;
        modf(rh, &rh_int);
        const long lobin = (long) rh_int - 1;
        if (hind == 0) hhlobin = lobin;
        for (int kk = 0; kk < numr; kk++)
            rind[kk] = (long) round(((hhlobin + kk * dr) * hfrac - lobin) * numbetween);
        rzw_volume_powers(data, numdata, numbetween, lobin, zh - numwid * hfrac * P_ACCEL_DZ,
                          zh + numwid * hfrac * P_ACCEL_DZ, numz, wh - numwid * hfrac * P_ACCEL_DW,
                          wh + numwid * hfrac * P_ACCEL_DW, numw, rind, numr, vp);
        for (size_t c = 0; c < ncell; c++) powsum[c] += vp[c] / locpow;
    }
    float maxpow = 0.0f;
    int wind = 0, zind = 0, rbest = 0;
    for (int ii = 0; ii < numw; ii++)
        for (int jj = 0; jj < numz; jj++)
            for (int kk = 0; kk < numr; kk++) {
                const float p = powsum[((size_t) ii * numz + jj) * numr + kk];
                if (p > maxpow) {
                    maxpow = p;
                    wind = ii;
                    zind = jj;
                    rbest = kk;
                }
            }
    free(powsum);
    free(vp);
    const double nh = numharm;
    *rout = (hhlobin + rbest * dr) / nh;
    *zout = ((zin * nh) - numwid * P_ACCEL_DZ + zind * P_ACCEL_DZ / (double) interpfac) / nh;
    *wout = ((win * nh) - numwid * P_ACCEL_DW + wind * P_ACCEL_DW / (double) interpfac) / nh;
    for (int ii = 0; ii < numharm; ii++) {
        const int hh = ii + 1;
        const double rr = *rout * hh, zz = *zout * hh, ww = *wout * hh;
        const float locpow = (float) orc_get_localpower3d(data, numdata, rr, zz, ww);
        orc_get_derivs3d(data, numdata, rr, zz, ww, locpow, &derivs[ii]);
        powers[ii] = derivs[ii].pow;
    }
}

/* optimize_accelcand (src/accel_utils.c:552-626) with harmonic polishing for
 * acceleration (jerk = 0) or jerk (jerk = 1) searches, OpenMP over
 * candidates; per candidate k the outputs hold ORC_MAX_HARM entries from
 * k * ORC_MAX_HARM. */
int orc_optimize_cands_w(const orc_fcomplex *fft, long long numbins, long long lobin, int ncand,
                         int jerk, const int *numharm, const double *r, const double *z,
                         const double *w, double *pows, double *hirs, double *hizs, double *hiws,
                         orc_rderivs *derivs, int nthreads)
{
    int bad = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1) reduction(| : bad)
#endif
    for (int k = 0; k < ncand; k++) {
        const int nh = numharm[k];
        const size_t o = (size_t) k * ORC_MAX_HARM;
        if (nh < 1 || nh > ORC_MAX_HARM) {
            bad = 1;
            continue;
        }
        double ro, zo, wo = 0.0;
        if (jerk)
            orc_max_rzw_arr_harmonics(fft, (long) numbins, nh, r[k] - (double) lobin, z[k], w[k], &ro,
                                      &zo, &wo, derivs + o, pows + o);
        else
            orc_max_rz_arr_harmonics(fft, (long) numbins, nh, r[k] - (double) lobin, z[k], &ro, &zo,
                                     derivs + o, pows + o);
        for (int ii = 0; ii < nh; ii++) {
            hirs[o + ii] = (ro + (double) lobin) * (ii + 1);
            hizs[o + ii] = zo * (ii + 1);
            hiws[o + ii] = jerk ? wo * (ii + 1) : 0.0;
        }
    }
    (void) nthreads;
    return bad ? -1 : 0;
}

/* calc_rzwerrs (src/characteristics.c:353-392). */
int orc_calc_rzwerrs(const orc_fourierprops *p, double T, orc_rzwerrs *o)
{
    if (T <= 0.0) return -1;
    double T2 = T * T, T3 = T2 * T;
    double r2 = p->r * p->r, sr2 = p->rerr * p->rerr, r4 = r2 * r2;
    double z2 = p->z * p->z, sz2 = p->zerr * p->zerr;
    double tmp = p->r * p->w - 3 * z2;
    o->f = p->r / T;
    o->ferr = p->rerr / T;
    o->fd = p->z / T2;
    o->fderr = p->zerr / T2;
    o->fdd = p->w / T3;
    o->fdderr = p->werr / T3;
    o->p = T / p->r;
    o->perr = T * p->rerr / r2;
    o->pd = -p->z / r2;
    o->pderr = sqrt(4 * z2 * sr2 / (r4 * r2) + sz2 / r4);
    if (p->w == 0.0)
        o->pdd = 0.0;
    else
        o->pdd = (2 * z2 - p->r * p->w) / (T * r2 * p->r);
    o->pdderr = sqrt((p->werr * p->werr * r4 + 16 * sz2 * r2 + 4 * tmp * tmp * sr2) / (r4 * r4 * T2));
    return 0;
}
