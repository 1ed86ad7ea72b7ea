/* FFTW stand-in for the reference's accelsearch program built by
 * oracle/build_ref.sh (declarations in oracle/refshim/fftw3.h).  Test
 * infrastructure only, written for this repository.
 *
 * Plans record the transform's geometry; execution copies the single-
 * precision input to double, runs a recursive mixed-radix decimation-in-time
 * DFT (any length: each level splits off the smallest prime factor and
 * combines with a per-plan table of exp(sign 2 pi i t / n)), and rounds the
 * unnormalised result to float, so in-place and out-of-place calls behave as
 * FFTW's.  Arithmetic is FP64 where FFTW's is FP32: results through it match
 * FFTW's to FP32 rounding, not bit for bit.  Wisdom calls do nothing. */
#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fftw3.h"

struct fftwf_plan_s {
    int n, howmany, istride, idist, ostride, odist, sign;
    fftwf_complex *in, *out;
    double complex *tw;            /* tw[t] = exp(sign 2 pi i t / n) */
};

void *fftwf_malloc(size_t n)
{
    void *p = NULL;
    if (posix_memalign(&p, 64, n ? n : 1)) return NULL;
    return p;
}

void fftwf_free(void *p) { free(p); }

int fftwf_import_system_wisdom(void) { return 0; }
int fftwf_import_wisdom_from_file(FILE *f) { (void) f; return 0; }
int fftwf_export_wisdom_to_file(FILE *f) { (void) f; return 0; }
int fftwf_alignment_of(float *p) { return (int) (((size_t) p) % 16); }

fftwf_plan fftwf_plan_guru_r2r(int rank, const fftwf_iodim *dims, int howmany_rank,
                               const fftwf_iodim *howmany_dims, float *in, float *out,
                               const fftwf_r2r_kind *kind, unsigned flags)
{
    (void) rank; (void) dims; (void) howmany_rank; (void) howmany_dims;
    (void) in; (void) out; (void) kind; (void) flags;
    fprintf(stderr, "FFTW stand-in: guru r2r plans are not provided\n");
    return NULL;
}

static fftwf_plan make_plan(int n, int howmany, fftwf_complex *in, int istride, int idist,
                            fftwf_complex *out, int ostride, int odist, int sign)
{
    if (n < 1 || howmany < 1) return NULL;
    fftwf_plan p = (fftwf_plan) calloc(1, sizeof *p);
    p->n = n;
    p->howmany = howmany;
    p->in = in;
    p->out = out;
    p->istride = istride;
    p->idist = idist;
    p->ostride = ostride;
    p->odist = odist;
    p->sign = sign < 0 ? -1 : 1;
    p->tw = (double complex *) malloc(sizeof(double complex) * n);
    for (long t = 0; t < n; t++) {
        const double ang = p->sign * 2.0 * M_PI * (double) t / (double) n;
        p->tw[t] = cos(ang) + I * sin(ang);
    }
    return p;
}

fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign,
                             unsigned flags)
{
    (void) flags;
    return make_plan(n, 1, in, 1, n, out, 1, n, sign);
}

fftwf_plan fftwf_plan_many_dft(int rank, const int *n, int howmany, fftwf_complex *in,
                               const int *inembed, int istride, int idist, fftwf_complex *out,
                               const int *onembed, int ostride, int odist, int sign,
                               unsigned flags)
{
    (void) inembed; (void) onembed; (void) flags;
    if (rank != 1) {
        fprintf(stderr, "FFTW stand-in: only rank-1 plans\n");
        return NULL;
    }
    return make_plan(n[0], howmany, in, istride, idist, out, ostride, odist, sign);
}

/* y[k] = sum_j x[j s] w^(j k T/m) for the m-point sub-transform whose input
 * is x with stride s; tw holds the n-point table, T = n / m. */
static void dft_rec(const double complex *x, long s, double complex *y, long m,
                    const double complex *tw, long n, double complex *scratch)
{
    if (m == 1) {
        y[0] = x[0];
        return;
    }
    long p = 2;
    while (m % p) p++;
    const long q = m / p;
    /* sub-transforms of the p decimated sequences, into scratch[j q + k] */
    for (long j = 0; j < p; j++)
        dft_rec(x + j * s, s * p, scratch + j * q, q, tw, n, y);
    const long T = n / m;
    for (long k = 0; k < q; k++)
        for (long r = 0; r < p; r++) {
            const long kk = k + r * q;
            double complex acc = 0.0;
            for (long j = 0; j < p; j++) acc += scratch[j * q + k] * tw[(j * kk * T) % n];
            y[kk] = acc;
        }
}

/* Work arrays per call: the reference executes one plan from several
   OpenMP threads (new-array execution is thread-safe in FFTW). */
static void run(const fftwf_plan p, fftwf_complex *in, fftwf_complex *out)
{
    const long n = p->n;
    double complex *a = (double complex *) malloc(sizeof(double complex) * 3 * n);
    double complex *b = a + n, *work = b + n;
    for (int h = 0; h < p->howmany; h++) {
        const fftwf_complex *src = in + (long) h * p->idist;
        for (long i = 0; i < n; i++)
            a[i] = (double) src[i * p->istride][0] + I * (double) src[i * p->istride][1];
        dft_rec(a, 1, b, n, p->tw, n, work);
        fftwf_complex *dst = out + (long) h * p->odist;
        for (long i = 0; i < n; i++) {
            dst[i * p->ostride][0] = (float) creal(b[i]);
            dst[i * p->ostride][1] = (float) cimag(b[i]);
        }
    }
    free(a);
}

void fftwf_execute(const fftwf_plan p)
{
    if (p) run(p, p->in, p->out);
}

void fftwf_execute_dft(const fftwf_plan p, fftwf_complex *in, fftwf_complex *out)
{
    if (p) run(p, in, out);
}

void fftwf_destroy_plan(fftwf_plan p)
{
    if (!p) return;
    free(p->tw);
    free(p);
}
