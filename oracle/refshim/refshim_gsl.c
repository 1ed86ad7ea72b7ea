/* GSL stand-in for the reference's accelsearch program built by
 * oracle/build_ref.sh (declarations in oracle/refshim/gsl/).  Test
 * infrastructure only, written for this repository.
 *
 *   gsl_cdf_chisq_Q/Qinv, gsl_cdf_gaussian_Q/Qinv  the oracle's restatements
 *       (oracle/accel_oracle.c: regularised incomplete gamma, erfc, inverse
 *       normal with Newton refinement; checked against scipy.special);
 *   gsl_stats_float_median  sorts the array in place (GSL also reorders it)
 *       and returns the middle value, or the mean of the two middle values
 *       in double for even n;
 *   gsl_vector_*            plain stride-1 vectors;
 *   nmsimplex2              Nelder & Mead (1965) as GSL's manual documents
 *       its nmsimplex2 minimiser: an initial simplex x0, x0 + step_i e_i;
 *       each iteration reflects the worst vertex through the centroid of the
 *       others, expands when the reflection beats the best vertex, else
 *       contracts that vertex halfway or, failing that, shrinks the simplex
 *       towards the best vertex; the size is the RMS distance of the vertices
 *       from their centroid, updated incrementally as vertices change and
 *       recomputed after a shrink (the manual's distinction from nmsimplex);
 *       vector norms as the reference BLAS dnrm2 (scaled sum of squares).
 *       Iterates agree with GSL's only to rounding;
 *   gsl_rng / gsl_ran       MT19937 with GSL's seeding, uniform and exponential
 *       variates (birdie zapping, -zaplist); no Gaussian variates. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gsl/gsl_errno.h"
#include "gsl/gsl_multimin.h"
#include "gsl/gsl_randist.h"
#include "gsl/gsl_statistics_float.h"
#include "gsl/gsl_vector.h"

double orc_chisq_q(double chi2, double dof);
double orc_chisq_qinv(double q, double dof);
double orc_gauss_q(double x);
double orc_gauss_qinv(double q);

double gsl_cdf_chisq_Q(double x, double nu) { return orc_chisq_q(x, nu); }
double gsl_cdf_chisq_Qinv(double Q, double nu) { return orc_chisq_qinv(Q, nu); }
double gsl_cdf_gaussian_Q(double x, double sigma) { return orc_gauss_q(x / sigma); }
double gsl_cdf_gaussian_Qinv(double Q, double sigma) { return sigma * orc_gauss_qinv(Q); }

static int cmp_float(const void *a, const void *b)
{
    const float x = *(const float *) a, y = *(const float *) b;
    return (x > y) - (x < y);
}

double gsl_stats_float_median(float data[], const size_t stride, const size_t n)
{
    if (n == 0) return 0.0;
    if (stride != 1) {
        fprintf(stderr, "GSL stand-in: median with stride %zu\n", stride);
        exit(1);
    }
    qsort(data, n, sizeof(float), cmp_float);
    const size_t lhs = (n - 1) / 2, rhs = n / 2;
    if (lhs == rhs) return data[lhs];
    return 0.5 * ((double) data[lhs] + (double) data[rhs]);
}

/* ---- vectors --------------------------------------------------------------- */
gsl_vector *gsl_vector_alloc(size_t n)
{
    gsl_vector *v = (gsl_vector *) calloc(1, sizeof *v);
    v->size = n;
    v->stride = 1;
    v->data = (double *) calloc(n ? n : 1, sizeof(double));
    v->owner = 1;
    return v;
}

void gsl_vector_free(gsl_vector *v)
{
    if (!v) return;
    free(v->data);
    free(v);
}

double gsl_vector_get(const gsl_vector *v, size_t i) { return v->data[i * v->stride]; }
void gsl_vector_set(gsl_vector *v, size_t i, double x) { v->data[i * v->stride] = x; }

void gsl_vector_set_all(gsl_vector *v, double x)
{
    for (size_t i = 0; i < v->size; i++) v->data[i * v->stride] = x;
}

/* ---- BLAS level 1 on plain arrays ------------------------------------------ */
static double nrm2(const double *x, size_t n)       /* reference BLAS dnrm2 */
{
    if (n == 1) return fabs(x[0]);
    double scale = 0.0, ssq = 1.0;
    for (size_t i = 0; i < n; i++)
        if (x[i] != 0.0) {
            const double ax = fabs(x[i]);
            if (scale < ax) {
                ssq = 1.0 + ssq * (scale / ax) * (scale / ax);
                scale = ax;
            } else {
                ssq += (ax / scale) * (ax / scale);
            }
        }
    return scale * sqrt(ssq);
}

static double dot(const double *x, const double *y, size_t n)
{
    double r = 0.0;
    for (size_t i = 0; i < n; i++) r += x[i] * y[i];
    return r;
}

static void axpy(double a, const double *x, double *y, size_t n)
{
    for (size_t i = 0; i < n; i++) y[i] += a * x[i];
}

/* ---- nmsimplex2 ------------------------------------------------------------ */
struct gsl_multimin_fminimizer_type {
    const char *name;
};
static const struct gsl_multimin_fminimizer_type nm2_type = {"nmsimplex2"};
const gsl_multimin_fminimizer_type *gsl_multimin_fminimizer_nmsimplex2 = &nm2_type;

typedef struct {
    size_t n, P;            /* dimension, vertices = n + 1 */
    double *x1;             /* P x n vertices */
    double *y1;             /* P values */
    double *center, *ws1, *ws2, *xc, *xc2;
    double S2;              /* squared size */
} nm2_state;

static double feval(gsl_multimin_function *f, const double *x, size_t n)
{
    gsl_vector v = {n, 1, (double *) x, NULL, 0};
    return f->f(&v, f->params);
}

static void centroid_of(nm2_state *s)
{
    memset(s->center, 0, sizeof(double) * s->n);
    for (size_t i = 0; i < s->P; i++) axpy(1.0, s->x1 + i * s->n, s->center, s->n);
    for (size_t j = 0; j < s->n; j++) s->center[j] *= 1.0 / (double) s->P;
}

static double rms_size(nm2_state *s)
{
    double ss = 0.0;
    for (size_t i = 0; i < s->P; i++) {
        memcpy(s->ws1, s->x1 + i * s->n, sizeof(double) * s->n);
        axpy(-1.0, s->center, s->ws1, s->n);
        const double t = nrm2(s->ws1, s->n);
        ss += t * t;
    }
    s->S2 = ss / (double) s->P;
    return sqrt(ss / (double) s->P);
}

/* the vertex `corner` moved along the line through the centroid of all
   vertices: coeff -1 reflects it through the centroid of the others, -2
   expands, 0.5 contracts it halfway towards that centroid */
static double trial_point(nm2_state *s, gsl_multimin_function *f, double coeff, size_t corner,
                          double *xc)
{
    const double P = (double) s->P;
    const double alpha = (1 - coeff) * P / (P - 1.0);
    const double beta = (P * coeff - 1.0) / (P - 1.0);
    memcpy(xc, s->center, sizeof(double) * s->n);
    for (size_t j = 0; j < s->n; j++) xc[j] *= alpha;
    axpy(beta, s->x1 + corner * s->n, xc, s->n);
    return feval(f, xc, s->n);
}

/* replaces vertex i, keeping the centroid and the squared size current
   without a full recomputation (the property that distinguishes nmsimplex2
   from nmsimplex in GSL's manual) */
static void replace_vertex(nm2_state *s, size_t i, const double *x, double val)
{
    const double P = (double) s->P;
    double *xo = s->x1 + i * s->n;
    memcpy(s->ws1, x, sizeof(double) * s->n);             /* delta = x - x_orig */
    axpy(-1.0, xo, s->ws1, s->n);
    memcpy(s->ws2, xo, sizeof(double) * s->n);            /* x_orig - centre */
    axpy(-1.0, s->center, s->ws2, s->n);
    const double d = nrm2(s->ws1, s->n);
    const double xmcd = dot(s->ws2, s->ws1, s->n);
    s->S2 += (2.0 / P) * xmcd + ((P - 1.0) / P) * (d * d / P);
    axpy(-1.0 / P, xo, s->center, s->n);
    axpy(1.0 / P, x, s->center, s->n);
    memcpy(xo, x, sizeof(double) * s->n);
    s->y1[i] = val;
}

/* every vertex but the best moves halfway towards it; centroid and size
   are recomputed */
static int shrink_to_best(nm2_state *s, gsl_multimin_function *f, size_t best)
{
    int status = GSL_SUCCESS;
    for (size_t i = 0; i < s->P; i++) {
        if (i == best) continue;
        for (size_t j = 0; j < s->n; j++)
            s->x1[i * s->n + j] = 0.5 * (s->x1[i * s->n + j] + s->x1[best * s->n + j]);
        s->y1[i] = feval(f, s->x1 + i * s->n, s->n);
        if (!isfinite(s->y1[i])) status = GSL_EBADFUNC;
    }
    centroid_of(s);
    rms_size(s);
    return status;
}

gsl_multimin_fminimizer *gsl_multimin_fminimizer_alloc(const gsl_multimin_fminimizer_type *T,
                                                       size_t n)
{
    gsl_multimin_fminimizer *m = (gsl_multimin_fminimizer *) calloc(1, sizeof *m);
    nm2_state *s = (nm2_state *) calloc(1, sizeof *s);
    m->type = T;
    m->x = gsl_vector_alloc(n);
    s->n = n;
    s->P = n + 1;
    s->x1 = (double *) calloc(s->P * n, sizeof(double));
    s->y1 = (double *) calloc(s->P, sizeof(double));
    s->center = (double *) calloc(n, sizeof(double));
    s->ws1 = (double *) calloc(n, sizeof(double));
    s->ws2 = (double *) calloc(n, sizeof(double));
    s->xc = (double *) calloc(n, sizeof(double));
    s->xc2 = (double *) calloc(n, sizeof(double));
    m->state = s;
    return m;
}

void gsl_multimin_fminimizer_free(gsl_multimin_fminimizer *m)
{
    if (!m) return;
    nm2_state *s = (nm2_state *) m->state;
    free(s->x1); free(s->y1); free(s->center); free(s->ws1); free(s->ws2);
    free(s->xc); free(s->xc2); free(s);
    gsl_vector_free(m->x);
    free(m);
}

int gsl_multimin_fminimizer_set(gsl_multimin_fminimizer *m, gsl_multimin_function *f,
                                const gsl_vector *x, const gsl_vector *step_size)
{
    nm2_state *s = (nm2_state *) m->state;
    const size_t n = s->n;
    if (x->size != n || step_size->size != n) return GSL_EINVAL;
    m->f = f;
    for (size_t j = 0; j < n; j++) m->x->data[j] = gsl_vector_get(x, j);
    double val = feval(f, m->x->data, n);
    if (!isfinite(val)) return GSL_EBADFUNC;
    memcpy(s->x1, m->x->data, sizeof(double) * n);
    s->y1[0] = val;
    for (size_t i = 0; i < n; i++) {
        memcpy(s->xc, m->x->data, sizeof(double) * n);
        s->xc[i] = m->x->data[i] + gsl_vector_get(step_size, i);
        val = feval(f, s->xc, n);
        if (!isfinite(val)) return GSL_EBADFUNC;
        memcpy(s->x1 + (i + 1) * n, s->xc, sizeof(double) * n);
        s->y1[i + 1] = val;
    }
    centroid_of(s);
    m->size = rms_size(s);
    return GSL_SUCCESS;
}

int gsl_multimin_fminimizer_iterate(gsl_multimin_fminimizer *m)
{
    nm2_state *s = (nm2_state *) m->state;
    gsl_multimin_function *f = m->f;
    size_t hi = 0, lo = 0, s_hi = 1;
    double dhi = s->y1[0], dlo = s->y1[0], ds_hi = s->y1[1];
    for (size_t i = 1; i < s->P; i++) {
        const double v = s->y1[i];
        if (v < dlo) {
            dlo = v;
            lo = i;
        } else if (v > dhi) {
            ds_hi = dhi;
            s_hi = hi;
            dhi = v;
            hi = i;
        } else if (v > ds_hi) {
            ds_hi = v;
            s_hi = i;
        }
    }
    (void) s_hi;
    const double val = trial_point(s, f, -1.0, hi, s->xc);
    if (isfinite(val) && val < s->y1[lo]) {
        const double val2 = trial_point(s, f, -2.0, hi, s->xc2);
        if (isfinite(val2) && val2 < s->y1[lo]) replace_vertex(s, hi, s->xc2, val2);
        else replace_vertex(s, hi, s->xc, val);
    } else if (!isfinite(val) || val > ds_hi) {
        if (isfinite(val) && val <= s->y1[hi]) replace_vertex(s, hi, s->xc, val);
        const double val2 = trial_point(s, f, 0.5, hi, s->xc2);
        if (isfinite(val2) && val2 <= s->y1[hi]) {
            replace_vertex(s, hi, s->xc2, val2);
        } else if (shrink_to_best(s, f, lo) != GSL_SUCCESS) {
            return GSL_FAILURE;
        }
    } else {
        replace_vertex(s, hi, s->xc, val);
    }
    size_t best = 0;
    for (size_t i = 1; i < s->P; i++)
        if (s->y1[i] < s->y1[best]) best = i;
    memcpy(m->x->data, s->x1 + best * s->n, sizeof(double) * s->n);
    m->fval = s->y1[best];
    m->size = s->S2 > 0 ? sqrt(s->S2) : rms_size(s);
    return GSL_SUCCESS;
}

double gsl_multimin_fminimizer_size(const gsl_multimin_fminimizer *m) { return m->size; }

int gsl_multimin_test_size(const double size, double epsabs)
{
    if (epsabs < 0.0) return GSL_EINVAL;
    return size < epsabs ? GSL_SUCCESS : GSL_CONTINUE;
}

/* ---- random numbers: MT19937 and the variates zapbirds draws ------------- */
/* MT19937 (Matsumoto & Nishimura, ACM TOMACS 8 (1998) 3-30) with the 2002
 * init_genrand seeding that GSL's gsl_rng_mt19937 documents (seed 0 means
 * 4357); gsl_rng_uniform is the 32-bit output / 2^32 and gsl_ran_exponential
 * -mu log1p(-u) (GSL 2.x).  Gaussian variates are not provided. */
static void no_rng(void)
{
    fprintf(stderr, "GSL stand-in: Gaussian variates are not provided\n");
    exit(1);
}

struct gsl_rng_type {
    const char *name;
};
struct gsl_rng {
    unsigned int s[624];
    int next;
};
static const struct gsl_rng_type mt_type = {"mt19937"};
const gsl_rng_type *gsl_rng_mt19937 = &mt_type;
const gsl_rng_type *gsl_rng_default = &mt_type;

void gsl_rng_set(const gsl_rng *r, unsigned long int seed)
{
    gsl_rng *m = (gsl_rng *) r;
    if (seed == 0) seed = 4357;
    m->s[0] = (unsigned int) (seed & 0xffffffffUL);
    for (int i = 1; i < 624; i++)
        m->s[i] = (unsigned int) (1812433253UL * (m->s[i - 1] ^ (m->s[i - 1] >> 30)) + i);
    m->next = 624;
}

gsl_rng *gsl_rng_alloc(const gsl_rng_type *T)
{
    (void) T;
    gsl_rng *r = (gsl_rng *) calloc(1, sizeof(gsl_rng));
    gsl_rng_set(r, 0);
    return r;
}

void gsl_rng_free(gsl_rng *r) { free(r); }

unsigned long int gsl_rng_get(const gsl_rng *r)
{
    gsl_rng *m = (gsl_rng *) r;
    if (m->next >= 624) {
        for (int k = 0; k < 624; k++) {
            unsigned int y = (m->s[k] & 0x80000000u) | (m->s[(k + 1) % 624] & 0x7fffffffu);
            m->s[k] = m->s[(k + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        m->next = 0;
    }
    unsigned int y = m->s[m->next++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

double gsl_rng_uniform(const gsl_rng *r) { return gsl_rng_get(r) / 4294967296.0; }
const gsl_rng_type *gsl_rng_env_setup(void) { return gsl_rng_default; }
double gsl_ran_gaussian(const gsl_rng *r, double sigma) { (void) r; (void) sigma; no_rng(); return 0.0; }
double gsl_ran_ugaussian(const gsl_rng *r) { (void) r; no_rng(); return 0.0; }
double gsl_ran_exponential(const gsl_rng *r, double mu) { return -mu * log1p(-gsl_rng_uniform(r)); }
