/*
 * ab_zap.c -- birdie zapping of accelsearch -zaplist (host C).
 *
 *   ab_read_zaplist   get_birdies        src/birdzap.c:6-88
 *   ab_zapbirds_host  the zapping loop   src/accelsearch.c:87-110 over
 *                     zapbirds           src/zapping.c:58-150 (noise mode)
 *
 * Each birdie's bins are replaced by noise with the local power level: the
 * median power of 200 bins on each side, 100 bins away from the birdie,
 * turned into a mean power (median / ln 2) and drawn as exponential powers
 * with uniform phases from GSL's MT19937 generator seeded with 1.  The
 * generator, its seeding and GSL's uniform and exponential variates are
 * restated here from their published definitions (Matsumoto & Nishimura,
 * ACM TOMACS 8 (1998) 3-30, with the 2002 init_genrand seeding GSL uses;
 * gsl_rng_uniform = the 32-bit output / 2^32; gsl_ran_exponential(mu) =
 * -mu log1p(-u) as in GSL 2.x).  The stream is sequential and the
 * replacement values go through the C library's sqrt / log1p / cos / sin as
 * the reference's do, so zapping runs on the host; on a device-resident
 * spectrum (ab_zapbirds, ab_series.cu) only the bins it reads and writes
 * cross the bus.  Each call starts a fresh stream at seed 1, as one
 * accelsearch run does.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "accel_b200.h"
#include "ab_host.h"

#define ZAP_MEDIANBINS 200                     /* src/zapping.c:7 */
#define ZAP_GUARDBINS (ZAP_MEDIANBINS / 2)     /* src/zapping.c:11 */
#define ZAP_SEED 1UL                           /* src/zapping.c:14 */
#define ZAP_TWOPI 6.2831853071795864769

/* ---- MT19937 ------------------------------------------------------------ */
enum { MT_N = 624, MT_M = 397 };

typedef struct {
    uint32_t s[MT_N];
    int next;
} mt_state;

static void mt_seed(mt_state *mt, unsigned long seed)
{
    if (seed == 0) seed = 4357;                /* GSL's default for seed 0 */
    mt->s[0] = (uint32_t) (seed & 0xffffffffUL);
    for (int i = 1; i < MT_N; i++)
        mt->s[i] = (uint32_t) (1812433253UL * (mt->s[i - 1] ^ (mt->s[i - 1] >> 30)) + (uint32_t) i);
    mt->next = MT_N;
}

static uint32_t mt_next(mt_state *mt)
{
    if (mt->next >= MT_N) {                    /* regenerate the whole state */
        for (int i = 0; i < MT_N; i++) {
            const uint32_t y = (mt->s[i] & 0x80000000u) | (mt->s[(i + 1) % MT_N] & 0x7fffffffu);
            mt->s[i] = mt->s[(i + MT_M) % MT_N] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        mt->next = 0;
    }
    uint32_t y = mt->s[mt->next++];
    y ^= y >> 11;                              /* tempering */
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

static double mt_uniform(mt_state *mt) { return mt_next(mt) / 4294967296.0; }

static double ran_exponential(mt_state *mt, double mu) { return -mu * log1p(-mt_uniform(mt)); }

unsigned int ab_mt19937_output(unsigned long seed, long long k)
{
    mt_state mt;
    mt_seed(&mt, seed);
    uint32_t v = 0;
    for (long long i = 0; i < k; i++) v = mt_next(&mt);
    return v;
}

/* ---- zap list ----------------------------------------------------------- */
static int cmp_lobin(const void *a, const void *b)
{
    const double x = ((const double *) a)[0], y = ((const double *) b)[0];
    return (x > y) - (x < y);
}

int ab_read_zaplist(const char *path, double T, double baryv, double *lobins, double *hibins,
                    int maxbirds, int *numbirds)
{
    if (!path || !numbirds || maxbirds < 0 || (maxbirds > 0 && (!lobins || !hibins)))
        return AB_ERR_ARG;
    FILE *f = fopen(path, "r");
    if (!f) return AB_ERR_ARG;
    char line[512];
    int n = 0, cap = 64;
    double *b = (double *) malloc(sizeof(double) * 2 * cap);
    if (!b) {
        fclose(f);
        return AB_ERR_NOMEM;
    }
    while (fgets(line, sizeof(line), f)) {
        double freq, width, lo, hi;
        if (line[0] == '#') continue;
        /* "B<freq> <width>": barycentric; otherwise topocentric, Doppler
           shifted by (1 + baryv) */
        if (line[0] == 'B') {
            if (sscanf(line + 1, "%lf %lf", &freq, &width) != 2) continue;
            lo = (freq - 0.5 * width) * T;
            hi = (freq + 0.5 * width) * T;
        } else {
            if (sscanf(line, "%lf %lf", &freq, &width) != 2) continue;
            lo = (freq - 0.5 * width) * T * (1.0 + baryv);
            hi = (freq + 0.5 * width) * T * (1.0 + baryv);
        }
        if (hi - lo < 1.0) {                   /* at least one bin wide */
            const double avg = 0.5 * (hi + lo);
            lo = avg - 0.5;
            hi = avg + 0.5;
        }
        if (n == cap) {
            double *nb = (double *) realloc(b, sizeof(double) * 4 * cap);
            if (!nb) {
                free(b);
                fclose(f);
                return AB_ERR_NOMEM;
            }
            b = nb;
            cap *= 2;
        }
        b[2 * n] = lo;
        b[2 * n + 1] = hi;
        n++;
    }
    fclose(f);
    qsort(b, (size_t) n, 2 * sizeof(double), cmp_lobin);
    for (int i = 0; i < n && i < maxbirds; i++) {
        lobins[i] = b[2 * i];
        hibins[i] = b[2 * i + 1];
    }
    free(b);
    *numbirds = n;
    return n > maxbirds ? AB_ERR_OVERFLOW : AB_OK;
}

/* ---- zapping ------------------------------------------------------------ */
static int cmp_float(const void *a, const void *b)
{
    const float x = *(const float *) a, y = *(const float *) b;
    return (x > y) - (x < y);
}

/* median of the powers of n bins (median(), src/median.c: GSL's float
   median, the mean of the two central values in double for even n) */
static float window_median(const ab_fcomplex *d, int n, float *scratch)
{
    for (int i = 0; i < n; i++) {
        volatile float a = d[i].r * d[i].r, b = d[i].i * d[i].i;   /* POWER(), no FMA */
        scratch[i] = a + b;
    }
    qsort(scratch, (size_t) n, sizeof(float), cmp_float);
    const int lhs = (n - 1) / 2, rhs = n / 2;
    if (lhs == rhs) return scratch[lhs];
    return (float) (0.5 * ((double) scratch[lhs] + (double) scratch[rhs]));
}

int ab_zap_bounds(long long numbins, long long N, const double *lobins, const double *hibins,
                  int numbirds, long long *span_lo, long long *span_hi)
{
    const double top = (double) (N / 2);
    long long lo = numbins, hi = 0;
    for (int i = 0; i < numbirds; i++) {
        if (lobins[i] >= top) break;
        const double hb = hibins[i] >= top ? top - 1 : hibins[i];
        const long long ilobin = (long long) floor(lobins[i]), ihibin = (long long) ceil(hb);
        if (ihibin - ilobin < 1) continue;
        /* the reference writes fft[ilobin .. ihibin) unchecked */
        if (ilobin < 0 || ihibin > numbins) return AB_ERR_ARG;
        long long a = ilobin - ZAP_GUARDBINS - ZAP_MEDIANBINS, b = ihibin + ZAP_GUARDBINS +
                                                                   ZAP_MEDIANBINS;
        if (a < 0) a = 0;
        if (b > numbins) b = numbins;
        if (a < lo) lo = a;
        if (b > hi) hi = b;
    }
    *span_lo = lo < hi ? lo : 0;
    *span_hi = lo < hi ? hi : 0;
    return AB_OK;
}

/* zapbirds(lobin, hibin, numbins, NULL, fft, 0) on span[k] = bin base + k */
static int zap_one(ab_fcomplex *span, long long base, long long numbins, double lobin,
                   double hibin, mt_state *mt, int *mt_ready)
{
    const long long ilobin = (long long) floor(lobin), ihibin = (long long) ceil(hibin);
    const long long binstozap = ihibin - ilobin;
    if (binstozap < 1) return 0;
    const long long lostart = ilobin - ZAP_GUARDBINS - ZAP_MEDIANBINS;
    const long long histart = ihibin + ZAP_GUARDBINS;
    const int uselo = lostart >= 1, usehi = histart + ZAP_MEDIANBINS <= numbins;
    if (!uselo && !usehi) return 0;            /* the reference warns and skips it */
    float scratch[ZAP_MEDIANBINS];
    float medpow = 0.0f;
    int numsides = 0;
    if (uselo) {
        medpow += window_median(span + (lostart - base), ZAP_MEDIANBINS, scratch);
        numsides++;
    }
    if (usehi) {
        medpow += window_median(span + (histart - base), ZAP_MEDIANBINS, scratch);
        numsides++;
    }
    medpow /= numsides;
    const float meanpow = medpow / -log(0.5);
    if (!*mt_ready) {
        mt_seed(mt, ZAP_SEED);
        *mt_ready = 1;
    }
    ab_fcomplex *d = span + (ilobin - base);
    for (long long i = 0; i < binstozap; i++) {
        const double amp = sqrt(ran_exponential(mt, meanpow));
        const double phase = ZAP_TWOPI * mt_uniform(mt);
        d[i].r = (float) (amp * cos(phase));
        d[i].i = (float) (amp * sin(phase));
    }
    return 1;
}

int ab_zapbirds_span(ab_fcomplex *span, long long base, long long numbins, long long N,
                     const double *lobins, const double *hibins, int numbirds, int *numzapped)
{
    mt_state mt;
    int mt_ready = 0, nz = 0;
    const double top = (double) (N / 2);       /* src/accelsearch.c:100 */
    for (int i = 0; i < numbirds; i++) {
        if (lobins[i] >= top) break;
        const double hi = hibins[i] >= top ? top - 1 : hibins[i];
        nz += zap_one(span, base, numbins, lobins[i], hi, &mt, &mt_ready);
    }
    if (numzapped) *numzapped = nz;
    return AB_OK;
}

int ab_zapbirds_host(ab_fcomplex *fft, long long numbins, long long N, const double *lobins,
                     const double *hibins, int numbirds, int *numzapped)
{
    if (!fft || numbins < 0 || numbirds < 0 || (numbirds > 0 && (!lobins || !hibins)))
        return AB_ERR_ARG;
    long long lo, hi;
    if (ab_zap_bounds(numbins, N, lobins, hibins, numbirds, &lo, &hi)) return AB_ERR_ARG;
    return ab_zapbirds_span(fft, 0, numbins, N, lobins, hibins, numbirds, numzapped);
}
