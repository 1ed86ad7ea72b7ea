/* Link-time stand-ins for the FFTW calls of the reference sources that
 * oracle/build_ref.sh compiles into oracle/_ref/libref_polish.so (the
 * polishing interpolators, responses and candidate properties).  Test
 * infrastructure only, written for this repository:
 *   fftwf_malloc / fftwf_free  plain malloc / free (include/vectors.h's
 *                              allocators call them);
 *   next2_to_n(x)              the smallest power of two >= x (declared in
 *                              include/misc_utils.h; src/misc_utils.c needs
 *                              the ERFA library);
 *   realfft(data, n, -1)       the forward real FFT of src/fastffts.c:163-246
 *                              (PRESTO's packing: n/2 complex bins, bin 0 holds
 *                              DC and Nyquist, negative exponent), computed in
 *                              FP64 by an iterative radix-2 transform and
 *                              rounded to float; n a power of two.  The
 *                              reference runs FFTW in FP32, so results through
 *                              it (gen_w_response) carry FFTW's boundary as an
 *                              FP64 stand-in, not FFTW's own rounding. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

void *fftwf_malloc(size_t n) { return malloc(n ? n : 1); }
void fftwf_free(void *p) { free(p); }

long long next2_to_n(long long x)
{
    long long p = 1;
    while (p < x) p *= 2;
    return p;
}

static void fft64(double *re, double *im, long n)
{
    for (long i = 1, j = 0; i < n; i++) {
        long bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j |= bit;
        if (i < j) {
            double t = re[i]; re[i] = re[j]; re[j] = t;
            t = im[i]; im[i] = im[j]; im[j] = t;
        }
    }
    for (long len = 2; len <= n; len <<= 1) {
        const double ang = -2.0 * M_PI / (double) len;
        for (long k = 0; k < len / 2; k++) {
            const double wr = cos(ang * k), wi = sin(ang * k);
            for (long s = 0; s < n; s += len) {
                const long a = s + k, b = a + len / 2;
                const double xr = re[b] * wr - im[b] * wi, xi = re[b] * wi + im[b] * wr;
                re[b] = re[a] - xr; im[b] = im[a] - xi;
                re[a] += xr; im[a] += xi;
            }
        }
    }
}

void realfft(float data[], long n, int isign)
{
    if (isign != -1 || n < 4 || (n & (n - 1))) {
        fprintf(stderr, "refshim realfft: only forward power-of-two transforms (n=%ld, isign=%d)\n",
                n, isign);
        exit(1);
    }
    double *re = malloc(sizeof(double) * n), *im = malloc(sizeof(double) * n);
    for (long i = 0; i < n; i++) { re[i] = data[i]; im[i] = 0.0; }
    fft64(re, im, n);
    data[0] = (float) re[0];
    data[1] = (float) re[n / 2];
    for (long k = 1; k < n / 2; k++) {
        data[2 * k] = (float) re[k];
        data[2 * k + 1] = (float) im[k];
    }
    free(re);
    free(im);
}
