/*
 * accel_oracle.c -- CPU restatement of PRESTO's accelsearch hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see accel_oracle.h).  Written from the
 * reference's behaviour; every routine cites the reference file:line that
 * it restates.  ORC_REAL selects the arithmetic of the plane generation
 * (double: FP64 oracle, float: FP32 like FFTW single precision).
 *
 * Pinned against the reference's own code, compiled from its unmodified
 * sources by oracle/build_ref.sh over stand-ins for FFTW / GSL / glib: the
 * f-fdot planes (tests/test_cpu_ref_planes.py, within 3.7e-7 of power + mean
 * power), the response generators, interpolators and candidate properties
 * (tests/test_cpu_ref_pins.py), and the reference program's output files
 * (tests/golden/ref_accel/, checked against the device).  What stays
 * unpinned is the third-party arithmetic itself (FFTW's FP32 rounding, GSL's
 * floating-point order).
 */
#include "accel_oracle.h"

#include <math.h>
#include <time.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef ORC_REAL
#define ORC_REAL double
#endif
typedef ORC_REAL real;

/* include/accel.h:19-35, include/presto.h:17-26,107, include/meminfo.h:2 */
#define A_NUMBETWEEN 2
#define A_DR 0.5
#define A_RDR 2
#define A_DZ 2
#define A_RDZ 0.5
#define A_DW 20
#define A_RDW 0.05
#define A_CLOSEST_R 15.0
#define NUMFINTBINS 16
#define DBLCORRECT 1e-14
#define MAXRAMUSE 2000000000LL
#define O_PI 3.14159265358979323846264338327950288
#define O_SQRT2 1.41421356237309504880168872420969808

/* ======================================================================
 * Geometry helpers
 * ==================================================================== */

/* src/accel_utils.c:36 -- round half away from zero, then truncate */
static int nearest_int(double x) { return (int) (x < 0 ? x - 0.5 : x + 0.5); }

static long long next2_to_n(long long x)          /* src/misc_utils.c:305-313 */
{
    long long i = 1;
    while (i < x) i <<= 1;
    return i;
}

int orc_next_good_fftlen(int n)                    /* src/corr_prep.c:3-16 */
{
    static const int lens[17] = {128, 192, 256, 384, 512, 768, 1024, 1280, 2048,
                                 4096, 5120, 7680, 10240, 12288, 15360, 16384, 25600};
    if (n <= lens[0]) return lens[0];
    if (n > lens[16]) return (int) next2_to_n(n);
    int i = 0;
    while (n > lens[i]) i++;
    return lens[i];
}

int orc_fftlen_from_kernwidth(int kw)              /* src/corr_prep.c:18-35 */
{
    if (kw < 6) return 128;
    if (kw < 52) return 256;
    if (kw < 67) return 512;
    if (kw < 378) return 1024;
    if (kw < 664) return 2048;
    if (kw < 1672) return 4096;
    if (kw < 3015) return 10240;
    if (kw < 3554) return 15360;
    if (kw < 6000) return 25600;
    return (int) next2_to_n((long long) kw * 5);
}

int orc_z_resp_halfwidth(double z)                 /* src/responses.c:27-47 (LOWACC) */
{
    return (int) (0.5 * 1.1 * fabs(z)) + NUMFINTBINS;
}

int orc_w_resp_halfwidth(double z, double w)       /* src/responses.c:49-84 (LOWACC) */
{
    if (fabs(w) < 1.0e-7) return orc_z_resp_halfwidth(z);
    double r0 = 0.5 * (w / 6.0 - z);
    double r1 = 0.5 * (w / 6.0 + z);
    double maxdev = fabs(r0) > fabs(r1) ? fabs(r0) : fabs(r1);
    double u_ext = 0.5 - z / w;
    if (u_ext > 0.0 && u_ext < 1.0) {
        double z0 = z - w / 2.0;
        double r_ext = 0.5 * w * u_ext * u_ext + z0 * u_ext + r0;
        maxdev = fabs(r_ext) > maxdev ? fabs(r_ext) : maxdev;
    }
    return (int) (1.1 * maxdev) + NUMFINTBINS;
}

double orc_calc_required_r(double f, double rfull)  /* src/accel_utils.c:54-60 */
{
    return rint(A_RDR * rfull * f) * A_DR;
}

int orc_calc_required_z(double f, double zfull)     /* src/accel_utils.c:63-69 */
{
    return nearest_int(A_RDZ * zfull * f) * A_DZ;
}

int orc_calc_required_w(double f, double wfull)     /* src/accel_utils.c:72-78 */
{
    return nearest_int(A_RDW * wfull * f) * A_DW;
}

static int index_from_r(double r, double lor) { return (int) ((r - lor) * A_RDR + DBLCORRECT); } /* :81-86 */
static int index_from_z(double z, double loz) { return (int) ((z - loz) * A_RDZ + DBLCORRECT); } /* :89-94 */
static int index_from_w(double w, double low) { return (int) ((w - low) * A_RDW + DBLCORRECT); } /* :97-102 */

static int twon_to_index(int n)                    /* src/accel_utils.c:42-51 */
{
    int x = 0;
    while (n > 1) { n >>= 1; x++; }
    return x;
}

/* src/accel_utils.c:1596-1805 (create_accelobs, hot-path geometry only) */
int orc_obs_init(const orc_params *p, orc_obs *obs)
{
    memset(obs, 0, sizeof(*obs));
    int zmax = p->zmax, wmax = p->wmax;
    if (zmax % A_DZ) zmax = (zmax / A_DZ + 1) * A_DZ;
    obs->N = p->N;
    obs->numbins = p->numbins;
    obs->nph = p->nph > 0 ? p->nph : 0.0f;
    obs->norm_type = (p->nph > 0 || !p->locpowP) ? 0 : 1;     /* src/accel_utils.c:1598-1620 */
    obs->noharmpolish = p->noharmpolishP ? 1 : 0;
    obs->lobin = p->lobin;
    if (obs->lobin > 0) {
        obs->nph = 0.0f;
        if (p->lobin > obs->numbins - 1) return -1;
    }
    int nh = p->numharm;
    if (nh != 1 && nh != 2 && nh != 4 && nh != 8 && nh != 16 && nh != 32) return -2;
    obs->numharmstages = twon_to_index(nh) + 1;
    obs->dz = A_DZ;
    obs->numz = (zmax / A_DZ) * 2 + 1;
    if (p->wmaxP) {
        if (wmax % A_DW) wmax = (wmax / A_DW + 1) * A_DW;
        obs->whi = wmax;
        obs->wlo = -wmax;
        obs->dw = A_DW;
        obs->numw = (wmax / A_DW) * 2 + 1;
        if (wmax == 0) obs->numw = 0;
    } else {
        obs->whi = obs->wlo = obs->dw = 0.0;
        obs->numw = 0;
    }
    obs->numbetween = A_NUMBETWEEN;
    obs->dt = p->dt;
    obs->T = p->dt * (double) p->N;
    if (p->floP) {
        obs->rlo = floor(p->flo * obs->T);
        if (obs->rlo < obs->lobin) obs->rlo = (double) obs->lobin;
        if (obs->rlo > obs->numbins - 1) return -3;
    } else {
        obs->rlo = p->rloP ? p->rlo : 1.0;
        if (obs->rlo < obs->lobin) obs->rlo = (double) obs->lobin;
        if (obs->rlo > obs->numbins - 1) return -3;
    }
    obs->highestbin = obs->numbins - 1;
    /* The reference leaves rhi unset when neither -fhi nor -rhi is given;
     * the clig defaults always set -fhi, so rhi = highestbin here. */
    obs->rhi = (double) obs->highestbin;
    if (p->fhiP) {
        obs->highestbin = (long long) ceil(p->fhi * obs->T);
        if (obs->highestbin > obs->numbins - 1) obs->highestbin = obs->numbins - 1;
        obs->rhi = (double) obs->highestbin;
        if (obs->highestbin < obs->rlo) return -4;
    } else if (p->rhiP) {
        obs->highestbin = (long long) p->rhi;
        if (obs->highestbin > obs->numbins - 1) obs->highestbin = obs->numbins - 1;
        obs->rhi = (double) obs->highestbin;
        if (obs->highestbin < obs->rlo) return -4;
    }
    obs->dr = A_DR;
    obs->zhi = zmax;
    obs->zlo = -zmax;
    obs->sigma = p->sigma;
    for (int ii = 0; ii < obs->numharmstages; ii++) {
        double nind;
        if (obs->numz == 1 && obs->numw == 0)
            nind = (obs->rhi - obs->rlo) / (1 << ii);
        else if (obs->numz > 1 && obs->numw == 0)
            nind = (obs->rhi - obs->rlo) * (obs->numz + 1) * (obs->dz / 6.95) / (1 << ii);
        else
            nind = (obs->rhi - obs->rlo) * (obs->numz + 1) * (obs->dz / 6.95) *
                   (obs->numw + 1) * (obs->dw / 44.2) / (1 << ii);
        obs->numindep[ii] = (long long) nind;
        obs->powcut[ii] = (float) orc_power_for_sigma(obs->sigma, 1 << ii,
                                                      (double) obs->numindep[ii]);
    }
    obs->maxkernlen = 2 * A_NUMBETWEEN * orc_w_resp_halfwidth(obs->zhi, obs->whi);
    obs->fftlen = orc_fftlen_from_kernwidth(obs->maxkernlen);
    if (obs->fftlen < 2048) obs->fftlen = 2048;
    obs->corr_uselen = obs->fftlen - obs->maxkernlen;
    if (obs->corr_uselen % A_RDR) obs->corr_uselen = obs->corr_uselen / A_RDR * A_RDR;
    obs->rstep = (int) (obs->corr_uselen * A_DR);
    long long memuse;
    if (p->wmaxP)
        memuse = 4LL * (obs->highestbin + obs->corr_uselen) * obs->numbetween * obs->numz * obs->numw;
    else
        memuse = 4LL * (obs->highestbin + obs->corr_uselen) * obs->numbetween * obs->numz;
    obs->inmem = (!p->wmaxP && (memuse < MAXRAMUSE || p->inmemP)) ? 1 : 0;
    return 0;
}

/* ======================================================================
 * Statistics (GSL boundary restated; checked against scipy.special)
 * ==================================================================== */

/* Regularised upper incomplete gamma Q(a,x): power series for x < a+1,
 * Lentz continued fraction otherwise (Numerical Recipes 2ed, 6.2). */
static double gamma_q(double a, double x)
{
    if (x <= 0.0) return 1.0;
    double gln = lgamma(a);
    if (x < a + 1.0) {
        double ap = a, sum = 1.0 / a, del = sum;
        for (int n = 0; n < 100000; n++) {
            ap += 1.0;
            del *= x / ap;
            sum += del;
            if (fabs(del) < fabs(sum) * 1e-17) break;
        }
        return 1.0 - sum * exp(-x + a * log(x) - gln);
    } else {
        const double fpmin = 1e-300;
        double b = x + 1.0 - a, c = 1.0 / fpmin, d = 1.0 / b, h = d;
        for (int i = 1; i < 100000; i++) {
            double an = -i * (i - a);
            b += 2.0;
            d = an * d + b;
            if (fabs(d) < fpmin) d = fpmin;
            c = b + an / c;
            if (fabs(c) < fpmin) c = fpmin;
            d = 1.0 / d;
            double del = d * c;
            h *= del;
            if (fabs(del - 1.0) < 1e-17) break;
        }
        return exp(-x + a * log(x) - gln) * h;
    }
}

double orc_chisq_q(double chi2, double dof) { return gamma_q(0.5 * dof, 0.5 * chi2); }

double orc_gauss_q(double x) { return 0.5 * erfc(x / O_SQRT2); }

/* Inverse of the upper normal tail: A&S 26.2.23 start, Newton on log Q. */
double orc_gauss_qinv(double q)
{
    if (q <= 0.0) return INFINITY;
    if (q >= 1.0) return -INFINITY;
    if (q > 0.5) return -orc_gauss_qinv(1.0 - q);
    double t = sqrt(-2.0 * log(q));
    double x = t - (2.515517 + t * (0.802853 + t * 0.010328)) /
                   (1.0 + t * (1.432788 + t * (0.189269 + t * 0.001308)));
    double lq = log(q);
    for (int it = 0; it < 50; it++) {
        double Q = orc_gauss_q(x);
        double lQ = log(Q);
        double pdf = exp(-0.5 * x * x) / sqrt(2.0 * O_PI);
        double step = (lQ - lq) / (pdf / Q);   /* d(lnQ)/dx = -pdf/Q */
        x += step;
        if (fabs(step) < 1e-15 * (fabs(x) + 1e-300)) break;
    }
    return x;
}

/* Inverse of the chi-square upper tail by safeguarded Newton on log Q. */
double orc_chisq_qinv(double q, double dof)
{
    double k = 0.5 * dof;
    double z = orc_gauss_qinv(q);
    double h = 2.0 / (9.0 * dof);
    double c = dof * pow(1.0 - h + z * sqrt(h), 3.0);   /* Wilson-Hilferty */
    if (!(c > 0.0)) c = dof;
    double lo = 0.0, hi = INFINITY, lq = log(q);
    for (int it = 0; it < 200; it++) {
        double Q = orc_chisq_q(c, dof);
        double lQ = log(Q);
        if (lQ > lq) lo = c; else hi = c;
        double lpdf = (k - 1.0) * log(c) - 0.5 * c - k * log(2.0) - lgamma(k);
        double step = (lQ - lq) / exp(lpdf - lQ);
        double cn = c + step;
        if (!(cn > lo && cn < hi)) cn = isinf(hi) ? 2.0 * c + 1.0 : 0.5 * (lo + hi);
        if (fabs(cn - c) < 1e-15 * c) { c = cn; break; }
        c = cn;
    }
    return c;
}

/* src/characteristics.c:399-416, A&S 26.2.23 */
static double extended_equiv_gaussian_sigma(double logp)
{
    double t = sqrt(-2.0 * logp);
    double num = 2.515517 + t * (0.802853 + t * 0.010328);
    double den = 1.0 + t * (1.432788 + t * (0.189269 + t * 0.001308));
    return t - num / den;
}

/* src/characteristics.c:419-437, A&S 6.5.32 */
static double log_asymtotic_incomplete_gamma(double a, double z)
{
    double x = 1.0, newxpart = 1.0, term = 1.0;
    int ii = 1;
    while (fabs(newxpart) > 1e-15) {
        term *= (a - ii);
        newxpart = term / pow(z, ii);
        x += newxpart;
        ii += 1;
    }
    return (a - 1.0) * log(z) - z + log(x);
}

/* src/characteristics.c:440-454, A&S 6.1.41 */
static double log_asymtotic_gamma(double z)
{
    double x = (z - 0.5) * log(z) - z + 0.91893853320467267;
    double y = 1.0 / (z * z);
    x += (((-5.9523809523809529e-4 * y + 7.9365079365079365079365e-4) * y -
           2.7777777777777777777778e-3) * y + 8.3333333333333333333333e-2) / z;
    return x;
}

double orc_equivalent_gaussian_sigma(double logp)  /* src/characteristics.c:459-470 */
{
    double x;
    if (logp < -600.0) x = extended_equiv_gaussian_sigma(logp);
    else x = orc_gauss_qinv(exp(logp));
    return (x < 0.0) ? 0.0 : x;
}

double orc_chi2_logp(double chi2, double dof)     /* src/characteristics.c:473-506 */
{
    if (chi2 <= 0.0) return -INFINITY;
    if (chi2 > 1200.0 || (dof > 30 && chi2 > 100.0))
        return log_asymtotic_incomplete_gamma(0.5 * dof, 0.5 * chi2) -
               log_asymtotic_gamma(0.5 * dof);
    return log(orc_chisq_q(chi2, dof));
}

double orc_candidate_sigma(double power, int numsum, double numtrials) /* :526-546 */
{
    if (power <= 0.0) return 0.0;
    double logp = orc_chi2_logp(2.0 * power, 2.0 * numsum);
    logp += log(numtrials);
    return orc_equivalent_gaussian_sigma(logp);
}

double orc_power_for_sigma(double sigma, int numsum, double numtrials) /* :549-559 */
{
    double q = orc_gauss_q(sigma) / numtrials;
    return 0.5 * orc_chisq_qinv(q, 2.0 * numsum);
}

/* src/median.c:6-12: GSL median (mean of the two central order statistics
 * for even n), restated as a full sort of a copy. */
static int cmp_float(const void *a, const void *b)
{
    float x = *(const float *) a, y = *(const float *) b;
    return (x > y) - (x < y);
}

float orc_median(float *arr, int n)
{
    if (n <= 0) return 0.0f;
    float *tmp = (float *) malloc(sizeof(float) * n);
    memcpy(tmp, arr, sizeof(float) * n);
    qsort(tmp, n, sizeof(float), cmp_float);
    double m;
    if (n & 1) m = tmp[n / 2];
    else m = 0.5 * ((double) tmp[(n - 1) / 2] + (double) tmp[n / 2]);
    free(tmp);
    return (float) m;
}

/* ======================================================================
 * Fresnel integrals: power series for small x, Lentz continued fraction of
 * erfc((1-i) sqrt(pi)/2 x) for large x (Numerical Recipes 2ed, 6.9).
 * Replaces Cephes fresnl() used at src/responses.c:291-292.
 * ==================================================================== */
void orc_fresnel(double xin, double *s, double *c)
{
    double x = fabs(xin);
    double S, C;
    if (x < 1e-300) {
        S = 0.0; C = 0.0;
    } else if (x <= 1.8) {
        /* C = sum (-1)^n (pi/2)^(2n) x^(4n+1)/((2n)!(4n+1)),
           S = sum (-1)^n (pi/2)^(2n+1) x^(4n+3)/((2n+1)!(4n+3)) */
        double t = 0.5 * O_PI * x * x;          /* (pi/2) x^2 */
        double term = x, sumc = 0.0, sums = 0.0;
        for (int k = 0; k < 200; k++) {        /* term = t^k x / k! with signs */
            double contrib = term / (2 * k + 1);
            if ((k & 1) == 0) {
                if ((k & 3) == 0) sumc += contrib; else sumc -= contrib;
            } else {
                if ((k & 3) == 1) sums += contrib; else sums -= contrib;
            }
            term *= t / (k + 1);
            if (fabs(term) < 1e-18 * (fabs(sumc) + fabs(sums)) && k > 4) break;
        }
        C = sumc; S = sums;
    } else {
        /* 2 z^2 = -i pi x^2 ;  erfc(z) = (1-i) x e^{i pi x^2/2} / K,
           K = b0 - a1/(b1 - a2/(b2 - ...)), b_n = 1 + 4n - i pi x^2,
           a_n = (2n-1)(2n);  C + iS = (1+i)/2 (1 - erfc(z)). */
        const double fpmin = 1e-300;
        double px2 = O_PI * x * x;
        double br = 1.0, bi = -px2;
        double cr = 1.0 / fpmin, ci = 0.0;
        double den = br * br + bi * bi;
        double dr = br / den, di = -bi / den;
        double hr = dr, hi = di;
        for (int n = 1; n < 100000; n++) {
            double an = -(double) (2 * n - 1) * (double) (2 * n);
            br += 4.0;
            /* d = 1/(an*d + b) */
            double tr = an * dr + br, ti = an * di + bi;
            den = tr * tr + ti * ti;
            dr = tr / den; di = -ti / den;
            /* c = b + an/c */
            den = cr * cr + ci * ci;
            double qr = an * cr / den, qi = -an * ci / den;
            cr = br + qr; ci = bi + qi;
            double delr = cr * dr - ci * di, deli = cr * di + ci * dr;
            double nhr = hr * delr - hi * deli, nhi = hr * deli + hi * delr;
            hr = nhr; hi = nhi;
            if (fabs(delr - 1.0) + fabs(deli) < 1e-16) break;
        }
        /* erfc = (1-i) x e^{i px2/2} * h */
        double ph = 0.5 * px2;
        double er = cos(ph), ei = sin(ph);
        double ar = x * (er + ei), ai = x * (ei - er);      /* (1-i) x e^{i ph} */
        double fr = ar * hr - ai * hi, fi = ar * hi + ai * hr;
        double gr = 1.0 - fr, gi = -fi;                      /* 1 - erfc */
        C = 0.5 * (gr - gi);
        S = 0.5 * (gr + gi);
    }
    if (xin < 0.0) { C = -C; S = -S; }
    *s = S; *c = C;
}

/* ======================================================================
 * Mixed-radix complex FFT (recursive decimation in time, radices 4,2,3,5
 * and generic), unnormalised, exp(sign*2*pi*i*j*k/n).
 * ==================================================================== */
typedef struct { real r, i; } rcplx;

typedef struct {
    int n, sign, nfac;
    int fac[64];          /* pairs (p, m) */
    rcplx *tw;            /* tw[j] = exp(sign 2 pi i j / n) */
} fftplan;

static void plan_init(fftplan *pl, int n, int sign)
{
    pl->n = n; pl->sign = sign; pl->nfac = 0;
    int m = n, p = 4;
    double fl = floor(sqrt((double) n));
    do {
        while (m % p) {
            switch (p) {
            case 4: p = 2; break;
            case 2: p = 3; break;
            default: p += 2; break;
            }
            if (p > fl) p = m;
        }
        m /= p;
        pl->fac[pl->nfac++] = p;
        pl->fac[pl->nfac++] = m;
    } while (m > 1);
    pl->tw = (rcplx *) malloc(sizeof(rcplx) * n);
    for (int j = 0; j < n; j++) {
        double ang = sign * 2.0 * O_PI * (double) j / (double) n;
        pl->tw[j].r = (real) cos(ang);
        pl->tw[j].i = (real) sin(ang);
    }
}

static inline rcplx cmul(rcplx a, rcplx b)
{
    rcplx c = {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r};
    return c;
}

static void fft_work(rcplx *out, const rcplx *in, int fstride, const int *fac,
                     const fftplan *pl)
{
    const int p = fac[0], m = fac[1];
    rcplx *out_beg = out;
    const rcplx *twid = pl->tw;
    if (m == 1) {
        for (int q = 0; q < p; q++) out[q] = in[q * fstride];
    } else {
        for (int q = 0; q < p; q++)
            fft_work(out + q * m, in + q * fstride, fstride * p, fac + 2, pl);
    }
    out = out_beg;
    if (p == 2) {
        for (int k = 0; k < m; k++) {
            rcplx t = cmul(out[k + m], twid[k * fstride]);
            rcplx a = out[k];
            out[k].r = a.r + t.r; out[k].i = a.i + t.i;
            out[k + m].r = a.r - t.r; out[k + m].i = a.i - t.i;
        }
    } else if (p == 4) {
        for (int k = 0; k < m; k++) {
            rcplx a0 = out[k];
            rcplx a1 = cmul(out[k + m], twid[k * fstride]);
            rcplx a2 = cmul(out[k + 2 * m], twid[2 * k * fstride]);
            rcplx a3 = cmul(out[k + 3 * m], twid[3 * k * fstride]);
            rcplx s0 = {a0.r + a2.r, a0.i + a2.i}, s1 = {a0.r - a2.r, a0.i - a2.i};
            rcplx s2 = {a1.r + a3.r, a1.i + a3.i}, s3 = {a1.r - a3.r, a1.i - a3.i};
            /* multiply s3 by sign*i */
            rcplx s3r;
            if (pl->sign < 0) { s3r.r = s3.i; s3r.i = -s3.r; }
            else { s3r.r = -s3.i; s3r.i = s3.r; }
            out[k].r = s0.r + s2.r; out[k].i = s0.i + s2.i;
            out[k + 2 * m].r = s0.r - s2.r; out[k + 2 * m].i = s0.i - s2.i;
            out[k + m].r = s1.r + s3r.r; out[k + m].i = s1.i + s3r.i;
            out[k + 3 * m].r = s1.r - s3r.r; out[k + 3 * m].i = s1.i - s3r.i;
        }
    } else {
        rcplx scratch[64];
        const int n = pl->n;
        for (int k = 0; k < m; k++) {
            for (int q = 0; q < p; q++)
                scratch[q] = q ? cmul(out[k + q * m], twid[(q * k * fstride) % n]) : out[k];
            for (int s = 0; s < p; s++) {
                rcplx acc = scratch[0];
                for (int q = 1; q < p; q++) {
                    int idx = (int) (((long long) q * s * m * fstride) % n);
                    rcplx t = cmul(scratch[q], twid[idx]);
                    acc.r += t.r; acc.i += t.i;
                }
                out[k + s * m] = acc;
            }
        }
    }
}

/* small plan cache; plans are created before any parallel region */
#define NPLANS 64
static fftplan g_plans[NPLANS];
static int g_nplans = 0;

static const fftplan *get_plan(int n, int sign)
{
    for (int i = 0; i < g_nplans; i++)
        if (g_plans[i].n == n && g_plans[i].sign == sign) return &g_plans[i];
    if (g_nplans >= NPLANS) { fprintf(stderr, "oracle: plan cache full\n"); abort(); }
    plan_init(&g_plans[g_nplans], n, sign);
    return &g_plans[g_nplans++];
}

static void cfft(rcplx *data, rcplx *tmp, int n, int sign)
{
    const fftplan *pl = get_plan(n, sign);
    fft_work(tmp, data, 1, pl->fac, pl);
    memcpy(data, tmp, sizeof(rcplx) * n);
}

/* Double-precision FFT used for templates (independent of ORC_REAL). */
typedef struct { double r, i; } dcplx;
static void dfft_rec(dcplx *out, const dcplx *in, int n, int stride, int sign)
{
    if (n == 1) { out[0] = in[0]; return; }
    int p = (n % 4 == 0) ? 4 : (n % 2 == 0) ? 2 : (n % 3 == 0) ? 3 : (n % 5 == 0) ? 5 : n;
    for (int f = 7; p == n && f * f <= n; f += 2)      /* else the smallest odd factor */
        if (n % f == 0) p = f;
    int m = n / p;
    for (int q = 0; q < p; q++) dfft_rec(out + q * m, in + q * stride, m, stride * p, sign);
    dcplx sc_small[64];
    dcplx *sc = p <= 64 ? sc_small : (dcplx *) malloc(sizeof(dcplx) * (size_t) p);
    for (int k = 0; k < m; k++) {
        for (int q = 0; q < p; q++) {
            double a = sign * 2.0 * O_PI * (double) q * k / n;
            double cr = cos(a), ci = sin(a);
            dcplx v = out[k + q * m];
            sc[q].r = v.r * cr - v.i * ci; sc[q].i = v.r * ci + v.i * cr;
        }
        for (int s = 0; s < p; s++) {
            dcplx acc = {0, 0};
            for (int q = 0; q < p; q++) {
                double a = sign * 2.0 * O_PI * (double) ((q * s) % p) / p;
                double cr = cos(a), ci = sin(a);
                acc.r += sc[q].r * cr - sc[q].i * ci;
                acc.i += sc[q].r * ci + sc[q].i * cr;
            }
            out[k + s * m] = acc;
        }
    }
    if (sc != sc_small) free(sc);
}

void orc_cfft_double(double *data, int n, int sign)
{
    dcplx *in = (dcplx *) malloc(sizeof(dcplx) * n);
    memcpy(in, data, sizeof(dcplx) * n);
    dfft_rec((dcplx *) data, in, n, 1, sign);
    free(in);
}

/* ======================================================================
 * Response templates
 * ==================================================================== */

/* src/responses.c:159-225: sinc response, written with direct sin/cos
 * instead of the trig recursion. */
static int gen_r_response_d(double roffset, int numbetween, int numkern, dcplx *out)
{
    if (roffset < 0.0 || roffset >= 1.0) return -1;
    if (numbetween < 1 || numbetween >= 20000) return -1;
    if (numkern < numbetween || numkern % (2 * numbetween)) return -1;
    double startr = O_PI * (numkern / (double) (2 * numbetween) + roffset);
    double delta = -O_PI / numbetween;
    for (int ii = 0; ii < numkern; ii++) {
        double r = startr + ii * delta;
        double s = sin(r), c = cos(r);
        double sinc = (r == 0.0) ? 1.0 : s / r;
        out[ii].r = c * sinc;
        out[ii].i = s * sinc;
    }
    if (roffset < 1E-3) {
        double t = roffset * roffset;
        out[numkern / 2].r = 1 - 6.579736267392905746 * t;
        out[numkern / 2].i = roffset * (O_PI - 10.335425560099940058 * t);
    }
    return 0;
}

/* src/responses.c:228-316: Fresnel-integral f-dot response */
static int gen_z_response_d(double roffset, int numbetween, double z, int numkern, dcplx *out)
{
    if (roffset < 0.0 || roffset >= 1.0) return -1;
    if (numbetween < 1 || numbetween >= 20000) return -1;
    if (numkern < numbetween || numkern % (2 * numbetween)) return -1;
    double absz = fabs(z);
    if (absz < 1E-4) return gen_r_response_d(roffset, numbetween, numkern, out);
    double startr = roffset - 0.5 * z, ip;
    double startroffset = (startr < 0) ? 1.0 + modf(startr, &ip) : modf(startr, &ip);
    int signz = (z < 0.0) ? -1 : 1;
    double zd = signz * O_SQRT2 / sqrt(absz);
    double cons = zd / 2.0;
    double pibyz = O_PI / z;
    startr += numkern / (double) (2 * numbetween);
    double delta = -1.0 / numbetween;
    for (int ii = 0; ii < numkern; ii++) {
        double r = startr + ii * delta;
        double yy = r * zd;
        double zz = yy + z * zd;
        double xx = pibyz * r * r;
        double c = cos(xx), s = sin(xx);
        double fsy, fcy, fsz, fcz;
        orc_fresnel(yy, &fsy, &fcy);
        orc_fresnel(zz, &fsz, &fcz);
        double tr = signz * (fcz - fcy);
        double ti = fsy - fsz;
        out[ii].r = (tr * c - ti * s) * cons;
        out[ii].i = -(tr * s + ti * c) * cons;
    }
    if (startroffset < 1E-3 && absz < 1E-3) {
        double zz = z * z, xx = startroffset * startroffset;
        int h = numkern / 2;
        out[h].r = 1.0 - 0.16449340668482264365 * zz;
        out[h].i = -0.5235987755982988731 * z;
        out[h].r += startroffset * 1.6449340668482264365 * z;
        out[h].i += startroffset * (O_PI - 0.5167712780049970029 * zz);
        out[h].r += xx * (-6.579736267392905746 + 0.9277056288952613070 * zz);
        out[h].i += xx * (3.1006276680299820175 * z);
    }
    return 0;
}

/* src/responses.c:333-418: f-dot-dot response by synthesising the chirp
 * and Fourier transforming it (here in FP64 throughout). */
static int gen_w_response_d(double roffset, int numbetween, double z, double w,
                            int numkern, dcplx *out)
{
    if (roffset < 0.0 || roffset >= 1.0) return -1;
    if (numbetween < 1 || numbetween >= 20000) return -1;
    if (numkern < numbetween || numkern % (2 * numbetween)) return -1;
    if (fabs(w) < 1E-4) return gen_z_response_d(roffset, numbetween, z, numkern, out);
    int npts = (int) next2_to_n(6 * orc_w_resp_halfwidth(z, w) + 200 + numkern / numbetween);
    double dt = 1.0 / (double) npts;
    double amp = 2.0 * dt;
    int fbar = npts / 4;
    double dfbar = (double) fbar + roffset;
    double f = dfbar - 0.5 * z + w / 12.0;
    double fd = (z - 0.5 * w) / 2.0;
    double fdd = w / 6.0;
    int nfft = npts * numbetween;
    dcplx *data = (dcplx *) calloc(nfft, sizeof(dcplx));
    for (int ii = 0; ii < npts; ii++) {
        double t = ii * dt;
        double phase = 2.0 * O_PI * (t * (t * (t * fdd + fd) + f));
        data[ii].r = amp * cos(phase);
    }
    orc_cfft_double((double *) data, nfft, -1);
    int first = fbar * numbetween - numkern / 2;
    for (int k = 0; k < numkern; k++) out[k] = data[first + k];
    free(data);
    return 0;
}

static int gen_resp_to_f(int kind, double roffset, int numbetween, double z, double w,
                         int numkern, orc_fcomplex *out)
{
    dcplx *tmp = (dcplx *) malloc(sizeof(dcplx) * numkern);
    int rc;
    if (kind == 0) rc = gen_r_response_d(roffset, numbetween, numkern, tmp);
    else if (kind == 1) rc = gen_z_response_d(roffset, numbetween, z, numkern, tmp);
    else rc = gen_w_response_d(roffset, numbetween, z, w, numkern, tmp);
    if (rc == 0)
        for (int i = 0; i < numkern; i++) {
            out[i].r = (float) tmp[i].r;
            out[i].i = (float) tmp[i].i;
        }
    free(tmp);
    return rc;
}

int orc_gen_r_response(double roffset, int numbetween, int numkern, orc_fcomplex *out)
{ return gen_resp_to_f(0, roffset, numbetween, 0, 0, numkern, out); }
int orc_gen_z_response(double roffset, int numbetween, double z, int numkern, orc_fcomplex *out)
{ return gen_resp_to_f(1, roffset, numbetween, z, 0, numkern, out); }
int orc_gen_w_response(double roffset, int numbetween, double z, double w, int numkern,
                       orc_fcomplex *out)
{ return gen_resp_to_f(2, roffset, numbetween, z, w, numkern, out); }

/* ======================================================================
 * Template banks: src/accel_utils.c:137-170 (calc_fftlen, init_kernel),
 * :202-237 (init_subharminfo)
 * ==================================================================== */
struct orc_bank {
    int numharm, harmnum, zmax, wmax, nz, nw, fftlen;
    int *hw;                 /* per template half width */
    rcplx *kern;             /* [nw][nz][fftlen], FFT'd */
    unsigned short *rinds, *zinds;
};

static int calc_fftlen(int numharm, int harmnum, int max_zfull, int max_wfull,
                       const orc_obs *obs)
{
    double f = (double) harmnum / (double) numharm;
    int bins_needed = (int) ceil(obs->corr_uselen * f) + 2;
    int end_effects = 2 * A_NUMBETWEEN *
        orc_w_resp_halfwidth(orc_calc_required_z(f, max_zfull), orc_calc_required_w(f, max_wfull));
    return orc_next_good_fftlen(bins_needed + end_effects);
}

orc_bank *orc_bank_create(const orc_obs *obs, int numharm, int harmnum)
{
    orc_bank *b = (orc_bank *) calloc(1, sizeof(orc_bank));
    double f = (double) harmnum / (double) numharm;
    b->numharm = numharm; b->harmnum = harmnum;
    b->zmax = orc_calc_required_z(f, (int) obs->zhi);
    b->wmax = orc_calc_required_w(f, (int) obs->whi);
    b->fftlen = (numharm == 1 && harmnum == 1) ? obs->fftlen
              : calc_fftlen(numharm, harmnum, (int) obs->zhi, (int) obs->whi, obs);
    b->nz = (b->zmax / A_DZ) * 2 + 1;
    b->nw = (b->wmax / A_DW) * 2 + 1;
    int L = b->fftlen, nt = b->nz * b->nw;
    b->hw = (int *) malloc(sizeof(int) * nt);
    b->kern = (rcplx *) malloc(sizeof(rcplx) * (size_t) nt * L);
    if (numharm > 1) {
        b->rinds = (unsigned short *) malloc(sizeof(unsigned short) * obs->corr_uselen);
        b->zinds = (unsigned short *) malloc(sizeof(unsigned short) * obs->corr_uselen);
    }
    for (int ii = 0; ii < b->nw; ii++) {
        for (int jj = 0; jj < b->nz; jj++) {
            int t = ii * b->nz + jj;
            int z = -b->zmax + jj * A_DZ, w = -b->wmax + ii * A_DW;
            int hw = orc_w_resp_halfwidth((double) z, (double) w);
            int numkern = 2 * A_NUMBETWEEN * hw;
            b->hw[t] = hw;
            dcplx *resp = (dcplx *) malloc(sizeof(dcplx) * numkern);
            gen_w_response_d(0.0, A_NUMBETWEEN, z, w, numkern, resp);
            /* src/corr_prep.c:92-114 place_complex_kernel: centre to index 0 */
            dcplx *placed = (dcplx *) calloc(L, sizeof(dcplx));
            int half = numkern / 2;
            memcpy(placed, resp + half, sizeof(dcplx) * half);
            memcpy(placed + L - half, resp, sizeof(dcplx) * half);
            orc_cfft_double((double *) placed, L, -1);
            rcplx *dst = b->kern + (size_t) t * L;
            for (int k = 0; k < L; k++) {
#if defined(ORC_FP32_TEMPLATES)
                dst[k].r = (real) (float) placed[k].r;
                dst[k].i = (real) (float) placed[k].i;
#else
                dst[k].r = (real) placed[k].r;
                dst[k].i = (real) placed[k].i;
#endif
            }
            free(placed);
            free(resp);
        }
    }
    return b;
}

void orc_bank_free(orc_bank *b)
{
    if (!b) return;
    free(b->hw); free(b->kern); free(b->rinds); free(b->zinds); free(b);
}

int orc_bank_info(const orc_bank *b, int *zmax, int *wmax, int *nz, int *nw, int *fftlen,
                  int *halfwidth)
{
    *zmax = b->zmax; *wmax = b->wmax; *nz = b->nz; *nw = b->nw; *fftlen = b->fftlen;
    *halfwidth = b->hw[0];
    return 0;
}

int orc_bank_kernel(const orc_bank *b, int wi, int zi, orc_fcomplex *out)
{
    if (wi < 0 || wi >= b->nw || zi < 0 || zi >= b->nz) return -1;
    const rcplx *src = b->kern + (size_t) (wi * b->nz + zi) * b->fftlen;
    for (int k = 0; k < b->fftlen; k++) { out[k].r = (float) src[k].r; out[k].i = (float) src[k].i; }
    return 0;
}

/* ======================================================================
 * Plane generation: src/accel_utils.c:993-1022 (get_fourier_amplitudes),
 * :1024-1198 (subharm_fderivs_vol)
 * ==================================================================== */
static void get_amplitudes(const orc_obs *obs, const orc_fcomplex *fft, long long lobin,
                           int numbins, orc_fcomplex *out)
{
    for (int i = 0; i < numbins; i++) {
        long long b = lobin + i - obs->lobin;
        if (b < 0 || b >= obs->numbins) { out[i].r = 0.0f; out[i].i = 0.0f; }
        else out[i] = fft[b];
    }
}

static double wall_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* thread-seconds spent in the correlation's FFTs since the last search's
   template banks were built (the CPU baseline reports the FFT share) */
static double g_t_fft;

static void fft_time_add(double s)
{
#ifdef _OPENMP
#pragma omp atomic
#endif
    g_t_fft += s;
}

int orc_subharm_fderivs_vol(const orc_obs *obs, const orc_fcomplex *fft, int numharm,
                            int harmnum, double fullrlo, double fullrhi, orc_bank *bank,
                            orc_ffdot *ffd)
{
    double f = (double) harmnum / (double) numharm;
    double drlo = orc_calc_required_r(f, fullrlo);
    double drhi = orc_calc_required_r(f, fullrhi);
    ffd->rlo = (long long) floor(drlo);
    ffd->zlo = orc_calc_required_z(f, obs->zlo);
    ffd->wlo = orc_calc_required_w(f, obs->wlo);
    if (numharm > 1 && !obs->inmem) {
        for (int ii = 0; ii < obs->corr_uselen; ii++) {
            double rr = fullrlo + ii * A_DR;
            double subr = orc_calc_required_r(f, rr);
            bank->rinds[ii] = (unsigned short) index_from_r(subr, (double) ffd->rlo);
        }
        for (int ii = 0; ii < obs->numz; ii++) {
            double zz = obs->zlo + ii * A_DZ;
            double subz = orc_calc_required_z(f, zz);
            bank->zinds[ii] = (unsigned short) index_from_z(subz, ffd->zlo);
        }
    }
    ffd->rinds = bank->rinds;
    ffd->zinds = bank->zinds;
    ffd->numrs = (int) ((ceil(drhi) - floor(drlo)) * A_RDR + DBLCORRECT) + 1;
    if (numharm == 1 && harmnum == 1) ffd->numrs = obs->corr_uselen;
    else if (ffd->numrs % A_RDR) ffd->numrs = (ffd->numrs / A_RDR + 1) * A_RDR;
    ffd->numzs = bank->nz;
    ffd->numws = bank->nw;

    const int binoffset = bank->hw[0];
    const int L = bank->fftlen;
    const long long lobin = ffd->rlo - binoffset;
    const int numdata = L / A_NUMBETWEEN;
    orc_fcomplex *data = (orc_fcomplex *) malloc(sizeof(orc_fcomplex) * numdata);
    get_amplitudes(obs, fft, lobin, numdata, data);

    /* normalisation (:1079-1115) */
    rcplx *pdata = (rcplx *) calloc(L, sizeof(rcplx));
    double norm;
    float *lnorm = NULL;            /* -locpow: per-bin factors */
    if (obs->nph > 0.0) {
        norm = 1.0 / sqrt(obs->nph);
    } else if (obs->norm_type == 1) {
        /* src/accel_utils.c:1100-1113: invsqrtf of corr_loc_pow per bin */
        float *pw = (float *) malloc(sizeof(float) * numdata);
        lnorm = (float *) malloc(sizeof(float) * numdata);
        for (int ii = 0; ii < numdata; ii++) {
            volatile float a = data[ii].r * data[ii].r;
            volatile float b = data[ii].i * data[ii].i;
            pw[ii] = a + b;
        }
        orc_loc_pow(pw, numdata, lnorm);
        for (int ii = 0; ii < numdata; ii++) lnorm[ii] = orc_invsqrtf(lnorm[ii]);
        free(pw);
        norm = 0.0;
    } else {
        float *pw = (float *) malloc(sizeof(float) * numdata);
        for (int ii = 0; ii < numdata; ii++) {
            volatile float a = data[ii].r * data[ii].r;   /* POWER() in float, no FMA */
            volatile float b = data[ii].i * data[ii].i;
            pw[ii] = a + b;
        }
        norm = 1.0 / sqrt(orc_median(pw, numdata) / log(2.0));
        free(pw);
    }
    /* spread_no_pad (src/corr_prep.c:62-74) */
    for (int ii = 0; ii < numdata && lnorm; ii++) {
        const float f = lnorm[ii];
        pdata[2 * ii].r = (real) (data[ii].r * f);          /* float products */
        pdata[2 * ii].i = (real) (data[ii].i * f);
    }
    for (int ii = 0; ii < numdata && !lnorm; ii++) {
#if defined(ORC_FP32_DATA)
        pdata[2 * ii].r = (real) (float) (data[ii].r * norm);
        pdata[2 * ii].i = (real) (float) (data[ii].i * norm);
#else
        pdata[2 * ii].r = (real) (data[ii].r * norm);
        pdata[2 * ii].i = (real) (data[ii].i * norm);
#endif
    }
    free(data);
    free(lnorm);
    rcplx *tmp = (rcplx *) malloc(sizeof(rcplx) * L);
    double tf0 = wall_s();
    cfft(pdata, tmp, L, -1);
    fft_time_add(wall_s() - tf0);
    free(tmp);
    get_plan(L, +1);

    const int nrs = ffd->numrs, nzs = ffd->numzs, nws = ffd->numws;
    ffd->powers = (float *) malloc(sizeof(float) * (size_t) nws * nzs * nrs);
    const int offset = binoffset * A_NUMBETWEEN;
    const real pnorm = (real) (1.0 / ((double) L * (double) L));
#ifdef _OPENMP
#pragma omp parallel
#endif
    {
        rcplx *buf = (rcplx *) malloc(sizeof(rcplx) * L);
        rcplx *out = (rcplx *) malloc(sizeof(rcplx) * L);
        const fftplan *pl = get_plan(L, +1);
        double t_fft = 0.0;
#ifdef _OPENMP
#pragma omp for collapse(2) schedule(static)
#endif
        for (int ii = 0; ii < nws; ii++) {
            for (int jj = 0; jj < nzs; jj++) {
                const rcplx *kern = bank->kern + (size_t) (ii * nzs + jj) * L;
                for (int kk = 0; kk < L; kk++) {          /* data * conj(kern) (:1167-1172) */
                    real dr = pdata[kk].r, di = pdata[kk].i;
                    real kr = kern[kk].r, ki = kern[kk].i;
                    buf[kk].r = dr * kr + di * ki;
                    buf[kk].i = di * kr - dr * ki;
                }
                const double tf = wall_s();
                fft_work(out, buf, 1, pl->fac, pl);      /* inverse FFT (:1174-1175) */
                t_fft += wall_s() - tf;
                float *op = ffd->powers + ((size_t) ii * nzs + jj) * nrs;
                for (int kk = 0; kk < nrs; kk++) {         /* powers (:1183-1188) */
                    const rcplx v = out[kk + offset];
                    op[kk] = (float) ((v.r * v.r + v.i * v.i) * pnorm);
                }
            }
        }
        free(buf); free(out);
        fft_time_add(t_fft);
    }
    free(pdata);
    return 0;
}

void orc_ffdot_free(orc_ffdot *f) { if (f && f->powers) { free(f->powers); f->powers = NULL; } }

/* src/accel_utils.c:1261-1282 */
void orc_add_ffdotpows(orc_ffdot *fund, const orc_ffdot *sub, int numharm, int harmnum)
{
    const double f = (double) harmnum / (double) numharm;
    for (int ii = 0; ii < fund->numws; ii++) {
        int ww = fund->wlo + ii * A_DW;
        int subw = orc_calc_required_w(f, ww);
        int wind = index_from_w(subw, sub->wlo);
        for (int jj = 0; jj < fund->numzs; jj++) {
            int zind = sub->zinds[jj];
            float *op = fund->powers + ((size_t) ii * fund->numzs + jj) * fund->numrs;
            const float *ip = sub->powers + ((size_t) wind * sub->numzs + zind) * sub->numrs;
            for (int kk = 0; kk < fund->numrs; kk++) op[kk] += ip[sub->rinds[kk]];
        }
    }
}

/* src/accel_utils.c:1219-1233 */
void orc_fund_to_ffdotplane(const orc_ffdot *ffd, const orc_obs *obs, float *plane)
{
    long long rlen = (obs->highestbin + obs->corr_uselen) * A_RDR;
    for (int ii = 0; ii < ffd->numzs; ii++)
        memcpy(plane + ii * rlen + ffd->rlo * A_RDR, ffd->powers + (size_t) ii * ffd->numrs,
               sizeof(float) * ffd->numrs);
}

/* src/accel_utils.c:1312-1361 */
void orc_inmem_add_ffdotpows(orc_ffdot *fund, const orc_obs *obs, const float *plane,
                             int numharm, int harmnum)
{
    const int rlo = (int) fund->rlo;
    const int numrs = fund->numrs, numzs = fund->numzs;
    const double f = (double) harmnum / (double) numharm;
    int *rinds = (int *) malloc(sizeof(int) * numrs);
    for (int ii = 0, rrint = A_RDR * rlo; ii < numrs; ii++, rrint++)
        rinds[ii] = (int) (rrint * f + 0.5);
    const long long rlen = (obs->highestbin + obs->corr_uselen) * A_RDR;
    for (int ii = 0; ii < numzs; ii++) {
        int zz = fund->zlo + ii * A_DZ;
        int subz = orc_calc_required_z(f, zz);
        int zind = index_from_z(subz, fund->zlo);
        const float *ip = plane + zind * rlen;
        float *op = fund->powers + (size_t) ii * numrs;
        for (int jj = 0; jj < numrs; jj++) op[jj] += ip[rinds[jj]];
    }
    free(rinds);
}

/* ======================================================================
 * Candidate list: src/accel_utils.c:387-469 (insert_new_accelcand)
 * ==================================================================== */
typedef struct onode { orc_cand c; struct onode *next; } onode;
struct orc_list { onode *head; };

orc_list *orc_list_new(void) { return (orc_list *) calloc(1, sizeof(orc_list)); }

void orc_list_free(orc_list *l)
{
    if (!l) return;
    onode *n = l->head;
    while (n) { onode *x = n->next; free(n); n = x; }
    free(l);
}

static onode *mknode(float power, float sigma, int numharm, double rr, double zz, double ww)
{
    onode *n = (onode *) calloc(1, sizeof(onode));
    n->c.power = power; n->c.sigma = sigma; n->c.numharm = numharm;
    n->c.r = rr; n->c.z = zz; n->c.w = ww;
    return n;
}

int orc_list_insert(orc_list *l, float power, float sigma, int numharm,
                    double rr, double zz, double ww)
{
    int added = 0;
    if (!l->head) { l->head = mknode(power, sigma, numharm, rr, zz, ww); return 1; }
    onode *tmp = l->head, *prev = NULL;
    double prev_diff_r = A_CLOSEST_R + 1.0, next_diff_r;
    while (tmp->next && tmp->c.r < rr) { prev = tmp; tmp = tmp->next; }
    next_diff_r = fabs(rr - tmp->c.r);
    if (prev) prev_diff_r = fabs(rr - prev->c.r);
    if (prev_diff_r < A_CLOSEST_R) {
        if (prev->c.sigma < sigma) {                 /* overwrite the prev cand */
            prev->c.power = power; prev->c.sigma = sigma; prev->c.numharm = numharm;
            prev->c.r = rr; prev->c.z = zz; prev->c.w = ww;
            added = 1;
        }
        if (next_diff_r < A_CLOSEST_R) {
            if (tmp->c.sigma < sigma) {
                if (added) {                 /* remove the next cand */
                    onode *p = l->head, *pp = NULL;
                    while (p && p != tmp) { pp = p; p = p->next; }
                    if (pp) pp->next = tmp->next; else l->head = tmp->next;
                    free(tmp);
                } else {
                    tmp->c.power = power; tmp->c.sigma = sigma; tmp->c.numharm = numharm;
                    tmp->c.r = rr; tmp->c.z = zz; tmp->c.w = ww;
                    added = 1;
                }
            }
        }
    } else if (next_diff_r < A_CLOSEST_R) {
        if (tmp->c.sigma < sigma) {
            tmp->c.power = power; tmp->c.sigma = sigma; tmp->c.numharm = numharm;
            tmp->c.r = rr; tmp->c.z = zz; tmp->c.w = ww;
            added = 1;
        }
    } else {
        onode *n = mknode(power, sigma, numharm, rr, zz, ww);
        added = 1;
        if (!tmp->next && tmp->c.r < (rr - A_CLOSEST_R)) { tmp->next = n; return added; }
        if (prev) { prev->next = n; n->next = tmp; }
        else { n->next = l->head; l->head = n; }
    }
    return added;
}

long long orc_list_get(const orc_list *l, orc_cand *out, long long maxout)
{
    long long n = 0;
    for (onode *p = l->head; p; p = p->next) {
        if (out && n < maxout) out[n] = p->c;
        n++;
    }
    return n;
}

/* src/accel_utils.c:1412-1452 (single-threaded visit order) */
void orc_search_ffdotpows(const orc_ffdot *ffd, int numharm, const orc_obs *obs,
                          orc_list *l, long long block, orc_hit *hits, long long maxhits,
                          long long *numhits)
{
    int stage = twon_to_index(numharm);
    float powcut = obs->powcut[stage];
    long long numindep = obs->numindep[stage];
    for (int ii = 0; ii < ffd->numws; ii++) {
        for (int jj = 0; jj < ffd->numzs; jj++) {
            const float *row = ffd->powers + ((size_t) ii * ffd->numzs + jj) * ffd->numrs;
            for (int kk = 0; kk < ffd->numrs; kk++) {
                float pow = row[kk];
                if (pow <= powcut) continue;
                if (hits && numhits) {
                    if (*numhits < maxhits) {
                        orc_hit *h = &hits[*numhits];
                        h->block = block; h->stage = stage; h->wi = ii; h->zi = jj; h->ri = kk;
                        h->power = pow;
                    }
                    (*numhits)++;
                }
                if (!l) continue;
                float sig = (float) orc_candidate_sigma(pow, numharm, (double) numindep);
                double rr = (ffd->rlo + kk * (double) A_DR) / (double) numharm;
                double zz = (ffd->zlo + jj * (double) A_DZ) / (double) numharm;
                double ww = (ffd->wlo + ii * (double) A_DW) / (double) numharm;
                orc_list_insert(l, pow, sig, numharm, rr, zz, ww);
            }
        }
    }
}

/* ======================================================================
 * Full search: src/accelsearch.c:161-224
 * ==================================================================== */
/* wall seconds of the last orc_accelsearch: template banks, then the block
   loop (timing for the CPU baseline, which needs no subtraction), and the
   thread-seconds its block loop spent inside the correlation FFTs */
static double g_t_setup, g_t_blocks, g_t_fft_blocks;
static int g_threads_used = 1;
static int g_loop_threads = 0;          /* block-loop threads; 0: as the banks */

void orc_set_loop_threads(int n) { g_loop_threads = n > 0 ? n : 0; }

void orc_last_timing(double *setup_s, double *blocks_s)
{
    *setup_s = g_t_setup;
    *blocks_s = g_t_blocks;
}

void orc_last_fft_share(double *fft_thread_s, double *loop_thread_s)
{
    *fft_thread_s = g_t_fft_blocks;
    *loop_thread_s = g_t_blocks * g_threads_used;
}

long long orc_accelsearch(const orc_params *p, const orc_fcomplex *fft, int nthreads,
                          long long first_block, long long max_blocks,
                          orc_cand *cands, long long maxcands,
                          orc_hit *hits, long long maxhits, long long *numhits,
                          long long *numblocks_done)
{
    return orc_accelsearch_sample(p, fft, nthreads, first_block, max_blocks, 1, cands,
                                  maxcands, hits, maxhits, numhits, numblocks_done);
}

long long orc_accelsearch_sample(const orc_params *p, const orc_fcomplex *fft, int nthreads,
                                 long long first_block, long long max_blocks,
                                 long long block_stride, orc_cand *cands, long long maxcands,
                                 orc_hit *hits, long long maxhits, long long *numhits,
                                 long long *numblocks_done)
{
    orc_obs obs;
    if (orc_obs_init(p, &obs)) return -1;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
    g_threads_used = omp_get_max_threads();
#else
    (void) nthreads;
    g_threads_used = 1;
#endif
    if (block_stride < 1) block_stride = 1;
    if (obs.inmem) block_stride = 1;        /* the plane needs every row */
    if (numhits) *numhits = 0;
    const double t0 = wall_s();
    const int stages = obs.numharmstages;
    orc_bank **banks = (orc_bank **) calloc(64, sizeof(orc_bank *));
    banks[0] = orc_bank_create(&obs, 1, 1);
    if (!obs.inmem)
        for (int s = 1; s < stages; s++)
            for (int h = 1; h < (1 << s); h += 2)
                banks[(1 << s) + h - 1] = orc_bank_create(&obs, 1 << s, h);
    float *plane = NULL;
    long long rlen = (obs.highestbin + obs.corr_uselen) * A_RDR;
    if (obs.inmem) plane = (float *) calloc((size_t) rlen * obs.numz, sizeof(float));
    const int rstep = obs.rstep;
    orc_list *l = orc_list_new();
    double startr, lastr, nextr;
#ifdef _OPENMP
    if (g_loop_threads > 0) {
        omp_set_num_threads(g_loop_threads);
        g_threads_used = g_loop_threads;
    }
#endif
    const double t1 = wall_s();
    g_t_setup = t1 - t0;
    g_t_fft = 0.0;
    if (obs.inmem) {
        startr = 8;
        while (startr < obs.rlo) {
            nextr = startr + rstep;
            lastr = nextr - A_DR;
            orc_ffdot fund;
            orc_subharm_fderivs_vol(&obs, fft, 1, 1, startr, lastr, banks[0], &fund);
            orc_fund_to_ffdotplane(&fund, &obs, plane);
            orc_ffdot_free(&fund);
            startr = nextr;
        }
    }
    startr = obs.rlo;
    long long block = 0, done = 0;
    while (startr + rstep < obs.highestbin) {
        if (max_blocks >= 0 && block >= first_block + max_blocks * block_stride) break;
        /* inmem: the plane needs all rows; a strided sample visits every
           block_stride-th block from first_block */
        int active = (block >= first_block && (block - first_block) % block_stride == 0) ||
                     obs.inmem;
        nextr = startr + rstep;
        lastr = nextr - A_DR;
        if (active) {
            orc_ffdot fund;
            orc_subharm_fderivs_vol(&obs, fft, 1, 1, startr, lastr, banks[0], &fund);
            int rec = block >= first_block && (block - first_block) % block_stride == 0;
            orc_search_ffdotpows(&fund, 1, &obs, rec ? l : NULL, block, rec ? hits : NULL,
                                 maxhits, numhits);
            if (stages > 1) {
                if (obs.inmem) orc_fund_to_ffdotplane(&fund, &obs, plane);
                for (int s = 1; s < stages; s++) {
                    int harmtosum = 1 << s;
                    for (int h = 1; h < harmtosum; h += 2) {
                        if (obs.inmem) {
                            orc_inmem_add_ffdotpows(&fund, &obs, plane, harmtosum, h);
                        } else {
                            orc_ffdot sub;
                            orc_subharm_fderivs_vol(&obs, fft, harmtosum, h, startr, lastr,
                                                    banks[harmtosum + h - 1], &sub);
                            orc_add_ffdotpows(&fund, &sub, harmtosum, h);
                            orc_ffdot_free(&sub);
                        }
                    }
                    orc_search_ffdotpows(&fund, harmtosum, &obs, rec ? l : NULL, block,
                                         rec ? hits : NULL, maxhits, numhits);
                }
            }
            orc_ffdot_free(&fund);
            if (rec) done++;
        }
        startr = nextr;
        block++;
    }
    g_t_blocks = wall_s() - t1;
    g_t_fft_blocks = g_t_fft;
    if (numblocks_done) *numblocks_done = done;
    long long nc = orc_list_get(l, cands, maxcands);
    orc_list_free(l);
    for (int i = 0; i < 64; i++) orc_bank_free(banks[i]);
    free(banks);
    free(plane);
    return nc;
}
