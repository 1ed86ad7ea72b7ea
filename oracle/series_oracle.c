/* series_oracle.c -- CPU restatement of accelsearch's time-series input path
 * (create_accelobs for .dat input, src/accel_utils.c:1516-1563): the forward
 * realfft (src/fastffts.c:163-246) and deredden (src/misc_utils.c:912-1067).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the device series-to-spectrum
 * kernels.  The reference's complex FFT is FFTW in single precision; here
 * it is the oracle's FP64 FFT rounded to float.  realfft's untangling uses
 * direct twiddles instead of the trig recursion (they agree to ~1e-13).
 * deredden is restated operation for operation in float (its fast inverse
 * square root included), so the same input gives the same output bits. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "accel_oracle.h"

#define S_TWOPI 6.28318530717958647692528676655900576

/* realfft(data, n, -1) (src/fastffts.c:163-229): n real samples in (any
 * even n), n/2 complex bins out in place, bin 0 = (DC, Nyquist). */
int orc_realfft_forward(float *data, long n)
{
    if (n < 4 || n % 2) return -1;
    const long nby2 = n >> 1, nby4 = n >> 2;
    double *d = (double *) malloc(sizeof(double) * (size_t) n);
    if (!d) return -1;
    for (long i = 0; i < n; i++) d[i] = data[i];
    orc_cfft_double(d, (int) nby2, -1);
    for (long i = 0; i < n; i++) data[i] = (float) d[i];
    free(d);
    orc_fcomplex *c = (orc_fcomplex *) data;
    const double cc = -0.5, theta = -S_TWOPI / (double) n;
    for (long il = 1, ih = nby2 - 1; il <= nby4; il++, ih--) {
        const double wr = cos(theta * il), wi = sin(theta * il);
        const double h1r = 0.5 * (c[il].r + c[ih].r), h1i = 0.5 * (c[il].i - c[ih].i);
        const double h2r = -cc * (c[il].i + c[ih].i), h2i = cc * (c[il].r - c[ih].r);
        const double h2rwr = h2r * wr, h2rwi = h2r * wi, h2iwr = h2i * wr, h2iwi = h2i * wi;
        c[il].r = (float) (h1r + h2rwr - h2iwi);
        c[il].i = (float) (h1i + h2iwr + h2rwi);
        c[ih].r = (float) (h1r - h2rwr + h2iwi);
        c[ih].i = (float) (-h1i + h2iwr + h2rwi);
    }
    const float t = c[0].r;
    c[0].r = t + c[0].i;
    c[0].i = t - c[0].i;
    return 0;
}

/* invsqrtf (src/misc_utils.c:291-302): the published fast inverse square
 * root (bit-level first guess, one Newton step), in float. */
float orc_invsqrtf(float x)
{
    union {
        float f;
        int32_t i;
    } t;
    t.f = x;
    t.i = 0x5f3759df - (t.i >> 1);
    const float y = t.f;
    return y * (1.5f - 0.5f * x * y * y);
}

static float block_mean(const orc_fcomplex *b, int n, float *pw)
{
    for (int ii = 0; ii < n; ii++) {
        const float pr = b[ii].r, pi = b[ii].i;
        pw[ii] = pr * pr + pi * pi;
    }
    return (float) ((double) orc_median(pw, n) / log(2.0));
}

/* deredden(fft, numbins, startwidth, endwidth, endfreq, T) on an in-memory
 * array (the mem adapters of src/misc_utils.c:1040-1067).  Returns the
 * number of bins written, or -1. */
long orc_deredden(orc_fcomplex *fft, long numbins, int startwidth, int endwidth, double endfreq,
                  double T)
{
    long rpos = 0, wpos = 0, binnum = 1, numwrote = 0;
    const float Tf = (float) T;
    const int cap = endwidth + 2;
    orc_fcomplex *bufa = (orc_fcomplex *) malloc(sizeof(orc_fcomplex) * cap);
    orc_fcomplex *bufb = (orc_fcomplex *) malloc(sizeof(orc_fcomplex) * cap);
    orc_fcomplex *out = (orc_fcomplex *) malloc(sizeof(orc_fcomplex) * cap);
    float *pw = (float *) malloc(sizeof(float) * cap);
    orc_fcomplex *oldbuf = bufa, *newbuf = bufb;
#define READB(buf, n)                                                                     \
    ({                                                                                    \
        long k_ = (n) < numbins - rpos ? (n) : numbins - rpos;                            \
        if (k_ < 0) k_ = 0;                                                               \
        memcpy((buf), fft + rpos, sizeof(orc_fcomplex) * k_);                             \
        rpos += k_;                                                                       \
        (int) k_;                                                                         \
    })
#define WRITEB(buf, n)                                                                    \
    do {                                                                                  \
        memcpy(fft + wpos, (buf), sizeof(orc_fcomplex) * (n));                            \
        wpos += (n);                                                                      \
    } while (0)
    long ret = -1;
    if (READB(oldbuf, 1) != 1) goto done;
    oldbuf[0].r = 1.0f;
    oldbuf[0].i = 0.0f;
    WRITEB(oldbuf, 1);
    numwrote += 1;
    int bufflen = startwidth;
    int nblk_old = READB(oldbuf, bufflen);
    if (nblk_old != bufflen) goto done;
    int mid_old = nblk_old / 2;
    float mean_old = block_mean(oldbuf, nblk_old, pw);
    float norm = orc_invsqrtf(mean_old), dslope = 1.0f;
    for (int ii = 0; ii < mid_old; ii++) {
        out[ii].r = oldbuf[ii].r * norm;
        out[ii].i = oldbuf[ii].i * norm;
    }
    WRITEB(out, mid_old);
    numwrote += mid_old;
    binnum += nblk_old;
    bufflen = (int) (startwidth * log((double) binnum));
    if (bufflen > endwidth) bufflen = endwidth;
    int nblk_new;
    while ((nblk_new = READB(newbuf, bufflen))) {
        const int mid_new = nblk_new / 2;
        const float mean_new = block_mean(newbuf, nblk_new, pw);
        dslope = (float) ((mean_new - mean_old) / (0.5 * (nblk_old + nblk_new)));
        int ii = 0, ind;
        for (ind = mid_old; ind < nblk_old; ii++, ind++) {
            norm = orc_invsqrtf(mean_old + dslope * ii);
            out[ii].r = oldbuf[ind].r * norm;
            out[ii].i = oldbuf[ind].i * norm;
        }
        for (ind = 0; ind < mid_new; ii++, ind++) {
            norm = orc_invsqrtf(mean_old + dslope * ii);
            out[ii].r = newbuf[ind].r * norm;
            out[ii].i = newbuf[ind].i * norm;
        }
        WRITEB(out, ii);
        numwrote += ii;
        binnum += nblk_new;
        if ((float) binnum / Tf < endfreq) {
            bufflen = (int) (startwidth * log((double) binnum));
            if (bufflen > endwidth) bufflen = endwidth;
        } else {
            bufflen = endwidth;
        }
        orc_fcomplex *tb = oldbuf;
        oldbuf = newbuf;
        newbuf = tb;
        nblk_old = nblk_new;
        mean_old = mean_new;
        mid_old = mid_new;
    }
    {
        int ii = 0;
        for (int ind = mid_old; ind < nblk_old; ii++, ind++) {
            norm = orc_invsqrtf(mean_old + dslope * ii);
            out[ii].r = oldbuf[ind].r * norm;
            out[ii].i = oldbuf[ind].i * norm;
        }
        WRITEB(out, nblk_old - mid_old);
        numwrote += nblk_old - mid_old;
    }
    ret = numwrote;
done:
#undef READB
#undef WRITEB
    free(bufa);
    free(bufb);
    free(out);
    free(pw);
    return ret;
}

/* corr_loc_pow (src/corr_routines.c:309-366): the powers correlated with a
 * double top-hat of 20 taps at +-6..+-15 bins, each (n / 2) / NUMLOCPOWAVG in
 * integer arithmetic, through real FFTs whose round trip (real_corr_conv,
 * src/correlations.c) carries 2 / n; the first and last 15 values take the
 * nearest value 15 from the edge.  Restated as the exact sum the FFTs
 * compute (they round it in FP32); no tap of a kept value wraps. */
void orc_loc_pow(const float *pw, int n, float *local)
{
    const int khw = 20 / 2 + 5;
    const double normal = (double) ((n / 2) / 20);
    for (int i = 0; i < n; i++) {
        const int c = i < khw ? khw : (i > n - 1 - khw ? n - 1 - khw : i);
        double s = 0.0;
        for (int j = 6; j <= khw; j++) s += (double) pw[c - j] + (double) pw[c + j];
        local[i] = (float) (s * normal * (2.0 / (double) n));
    }
}
