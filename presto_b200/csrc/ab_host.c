/*
 * ab_host.c -- host C side of the engine: search geometry and thresholds
 * (create_accelobs), template-bank geometry (create_subharminfos),
 * statistics (candidate_sigma / power_for_sigma), and the candidate list
 * with the replay of device threshold crossings in reference order.
 */
#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <unistd.h>
#include <sys/mman.h>

#include "ab_host.h"
#include "ab_index.h"

#define AB_MAXRAMUSE 2000000000LL      /* include/meminfo.h:2 */
#define AB_PI 3.14159265358979323846264338327950288
#define AB_SQRT2 1.41421356237309504880168872420969808

static long long next_pow2(long long x)                /* src/misc_utils.c:305-313 */
{
    long long i = 1;
    while (i < x) i <<= 1;
    return i;
}

int ab_next_good_fftlen(int n)                          /* src/corr_prep.c:3-16 */
{
    static const int good[17] = {128, 192, 256, 384, 512, 768, 1024, 1280, 2048,
                                 4096, 5120, 7680, 10240, 12288, 15360, 16384, 25600};
    if (n <= good[0]) return good[0];
    if (n > good[16]) return (int) next_pow2(n);
    int i = 0;
    while (n > good[i]) i++;
    return good[i];
}

int ab_fftlen_from_kernwidth(int kw)                    /* src/corr_prep.c:18-35 */
{
    static const int lim[9] = {6, 52, 67, 378, 664, 1672, 3015, 3554, 6000};
    static const int len[9] = {128, 256, 512, 1024, 2048, 4096, 10240, 15360, 25600};
    for (int i = 0; i < 9; i++)
        if (kw < lim[i]) return len[i];
    return (int) next_pow2((long long) kw * 5);
}

int ab_w_resp_halfwidth(double z, double w)             /* src/responses.c:27-84 */
{
    return ab_resp_halfwidth(z, w);
}

/* ------------------------------------------------------------------ */
/* statistics                                                          */
/* ------------------------------------------------------------------ */

/* Upper regularised incomplete gamma for the chi-square tail.  Every
 * search uses dof = 2*numsum, for which Q is the finite Poisson sum
 * exp(-x) sum_{j<k} x^j/j!; other dof use a continued fraction. */
static double chisq_upper(double chi2, double dof)
{
    double x = 0.5 * chi2, a = 0.5 * dof;
    if (x <= 0.0) return 1.0;
    if (a == floor(a) && a <= 512) {
        int k = (int) a;
        double term = 1.0, sum = 1.0;
        for (int j = 1; j < k; j++) { term *= x / j; sum += term; }
        return exp(-x + log(sum));
    }
    double gln = lgamma(a);
    if (x < a + 1.0) {
        double ap = a, s = 1.0 / a, d = s;
        for (int n = 0; n < 100000 && fabs(d) > fabs(s) * 1e-17; n++) { ap += 1; d *= x / ap; s += d; }
        return 1.0 - s * exp(-x + a * log(x) - gln);
    }
    double b = x + 1.0 - a, c = 1e300, d = 1.0 / b, h = d;
    for (int i = 1; i < 100000; i++) {
        double an = -i * (i - a);
        b += 2.0;
        d = an * d + b; if (fabs(d) < 1e-300) d = 1e-300;
        c = b + an / c; if (fabs(c) < 1e-300) c = 1e-300;
        d = 1.0 / d;
        double del = d * c;
        h *= del;
        if (fabs(del - 1.0) < 1e-17) break;
    }
    return exp(-x + a * log(x) - gln) * h;
}

static double gauss_upper(double x) { return 0.5 * erfc(x / AB_SQRT2); }

/* x with Q(x) = q for the standard normal upper tail, by Newton steps on
 * log Q from the Abramowitz & Stegun 26.2.23 starting value. */
static double gauss_upper_inv(double q)
{
    if (q <= 0.0) return INFINITY;
    if (q >= 1.0) return -INFINITY;
    if (q > 0.5) return -gauss_upper_inv(1.0 - q);
    double t = sqrt(-2.0 * log(q));
    double x = t - (2.515517 + t * (0.802853 + t * 0.010328)) /
                   (1.0 + t * (1.432788 + t * (0.189269 + t * 0.001308)));
    double lq = log(q);
    for (int it = 0; it < 60; it++) {
        double Q = gauss_upper(x);
        double dx = (log(Q) - lq) * Q / (exp(-0.5 * x * x) / sqrt(2.0 * AB_PI));
        x += dx;
        if (fabs(dx) <= 1e-15 * fabs(x)) break;
    }
    return x;
}

/* chi2 with Q(chi2; dof) = q: bracketed Newton on log Q. */
static double chisq_upper_inv(double q, double dof)
{
    double k = 0.5 * dof, z = gauss_upper_inv(q), h = 2.0 / (9.0 * dof);
    double c = dof * pow(1.0 - h + z * sqrt(h), 3.0);
    if (!(c > 0.0)) c = dof;
    double lo = 0.0, hi = INFINITY, lq = log(q);
    for (int it = 0; it < 300; it++) {
        double lQ = log(chisq_upper(c, dof));
        if (lQ > lq) lo = c; else hi = c;
        double lpdf = (k - 1.0) * log(c) - 0.5 * c - k * log(2.0) - lgamma(k);
        double cn = c + (lQ - lq) / exp(lpdf - lQ);
        if (!(cn > lo && cn < hi)) cn = isinf(hi) ? 2.0 * c + 1.0 : 0.5 * (lo + hi);
        if (fabs(cn - c) <= 1e-15 * c) { c = cn; break; }
        c = cn;
    }
    return c;
}

/* A&S 6.5.32 asymptotic log upper incomplete gamma (src/characteristics.c:419-437);
 * the series terminates for integer a. */
static double log_asym_inc_gamma(double a, double z)
{
    double x = 1.0, part = 1.0, term = 1.0;
    for (int i = 1; fabs(part) > 1e-15; i++) {
        term *= (a - i);
        part = term / pow(z, i);
        x += part;
    }
    return (a - 1.0) * log(z) - z + log(x);
}

/* A&S 6.1.41 Stirling series (src/characteristics.c:440-454). */
static double log_asym_gamma(double z)
{
    double x = (z - 0.5) * log(z) - z + 0.91893853320467267;
    double y = 1.0 / (z * z);
    x += (((-5.9523809523809529e-4 * y + 7.9365079365079365079365e-4) * y -
           2.7777777777777777777778e-3) * y + 8.3333333333333333333333e-2) / z;
    return x;
}

double ab_chi2_logp(double chi2, double dof)            /* src/characteristics.c:473-506 */
{
    if (chi2 <= 0.0) return -INFINITY;
    if (chi2 > 1200.0 || (dof > 30 && chi2 > 100.0))
        return log_asym_inc_gamma(0.5 * dof, 0.5 * chi2) - log_asym_gamma(0.5 * dof);
    return log(chisq_upper(chi2, dof));
}

double ab_equivalent_gaussian_sigma(double logp)        /* src/characteristics.c:399-470 */
{
    double x;
    if (logp < -600.0) {
        double t = sqrt(-2.0 * logp);
        x = t - (2.515517 + t * (0.802853 + t * 0.010328)) /
                (1.0 + t * (1.432788 + t * (0.189269 + t * 0.001308)));
    } else {
        x = gauss_upper_inv(exp(logp));
    }
    return (x < 0.0) ? 0.0 : x;
}

double ab_candidate_sigma(double power, int numsum, double numtrials)
{
    if (power <= 0.0) return 0.0;
    double logp = ab_chi2_logp(2.0 * power, 2.0 * numsum) + log(numtrials);
    return ab_equivalent_gaussian_sigma(logp);
}

double ab_power_for_sigma(double sigma, int numsum, double numtrials)
{
    double q = gauss_upper(sigma) / numtrials;
    return 0.5 * chisq_upper_inv(q, 2.0 * numsum);
}

/* ------------------------------------------------------------------ */
/* geometry                                                            */
/* ------------------------------------------------------------------ */

void ab_params_default(ab_params *p)                    /* src/accelsearch_cmd.c:22-61 */
{
    memset(p, 0, sizeof(*p));
    p->zmax = 200;
    p->numharm = 8;
    p->sigma = 2.0f;
    p->flo = 1.0; p->floP = 1;
    p->fhi = 10000.0; p->fhiP = 1;
}

static int twon_to_index(int n)
{
    int x = 0;
    while (n > 1) { n >>= 1; x++; }
    return x;
}

int ab_obs_init(const ab_params *p, ab_obs *obs)        /* src/accel_utils.c:1596-1805 */
{
    if (!p || !obs) return AB_ERR_ARG;
    memset(obs, 0, sizeof(*obs));
    if (p->N <= 0 || p->dt <= 0.0 || p->numbins <= 0) return AB_ERR_ARG;
    int zmax = p->zmax, wmax = p->wmax;
    if (zmax < 0 || wmax < 0) return AB_ERR_ARG;
    if (zmax % AB_DZ) zmax = (zmax / AB_DZ + 1) * AB_DZ;
    obs->N = p->N;
    obs->numbins = p->numbins;
    obs->nph = p->nph > 0.0f ? p->nph : 0.0f;
    /* -photon takes precedence; otherwise -locpow selects the local-power
     * normalisation (src/accel_utils.c:1598-1620) */
    obs->norm_type = (p->nph > 0.0f || !p->locpowP) ? 0 : 1;
    obs->noharmpolish = p->noharmpolishP ? 1 : 0;
    obs->lobin = p->lobin;
    if (obs->lobin > 0) {
        obs->nph = 0.0f;
        if (p->lobin > obs->numbins - 1) return AB_ERR_ARG;
    }
    int nh = p->numharm;
    if (nh != 1 && nh != 2 && nh != 4 && nh != 8 && nh != 16 && nh != 32) return AB_ERR_ARG;
    obs->numharmstages = twon_to_index(nh) + 1;
    obs->dz = AB_DZ;
    obs->numz = (zmax / AB_DZ) * 2 + 1;
    if (p->wmaxP) {
        if (wmax % AB_DW) wmax = (wmax / AB_DW + 1) * AB_DW;
        obs->whi = wmax;
        obs->wlo = -wmax;
        obs->dw = AB_DW;
        obs->numw = (wmax / AB_DW) * 2 + 1;
        if (wmax == 0) obs->numw = 0;
    }
    obs->numbetween = AB_NUMBETWEEN;
    obs->dt = p->dt;
    obs->T = p->dt * (double) p->N;
    if (p->floP) {
        obs->rlo = floor(p->flo * obs->T);
    } else {
        obs->rlo = p->rloP ? p->rlo : 1.0;
    }
    if (obs->rlo < obs->lobin) obs->rlo = (double) obs->lobin;
    if (obs->rlo > obs->numbins - 1) return AB_ERR_ARG;
    obs->highestbin = obs->numbins - 1;
    obs->rhi = (double) obs->highestbin;   /* left unset by the reference without -fhi/-rhi */
    if (p->fhiP || p->rhiP) {
        obs->highestbin = p->fhiP ? (long long) ceil(p->fhi * obs->T) : (long long) p->rhi;
        if (obs->highestbin > obs->numbins - 1) obs->highestbin = obs->numbins - 1;
        obs->rhi = (double) obs->highestbin;
        if (obs->highestbin < obs->rlo) return AB_ERR_ARG;
    }
    obs->dr = AB_DR;
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
        obs->powcut[ii] = (float) ab_power_for_sigma(obs->sigma, 1 << ii,
                                                     (double) obs->numindep[ii]);
    }
    obs->maxkernlen = 2 * AB_NUMBETWEEN * ab_w_resp_halfwidth(obs->zhi, obs->whi);
    obs->fftlen = ab_fftlen_from_kernwidth(obs->maxkernlen);
    if (obs->fftlen < 2048) obs->fftlen = 2048;
    obs->corr_uselen = obs->fftlen - obs->maxkernlen;
    if (obs->corr_uselen % AB_RDR) obs->corr_uselen = obs->corr_uselen / AB_RDR * AB_RDR;
    if (obs->corr_uselen <= 0 || obs->corr_uselen >= 65536) return AB_ERR_ARG;
    obs->rstep = (int) (obs->corr_uselen * AB_DR);
    long long memuse = 4LL * (obs->highestbin + obs->corr_uselen) * obs->numbetween * obs->numz;
    if (p->wmaxP) memuse *= obs->numw;
    obs->inmem = (!p->wmaxP && (memuse < AB_MAXRAMUSE || p->inmemP)) ? 1 : 0;
    return AB_OK;
}

long long ab_num_blocks(const ab_obs *obs)             /* src/accelsearch.c:187-224 */
{
    long long n = 0;
    double startr = obs->rlo;
    while (startr + obs->rstep < obs->highestbin) { n++; startr += obs->rstep; }
    return n;
}

long long ab_num_preblocks(const ab_obs *obs)          /* src/accelsearch.c:166-183 */
{
    if (!obs->inmem) return 0;
    long long n = 0;
    double startr = 8;
    while (startr < obs->rlo) { n++; startr += obs->rstep; }
    return n;
}

void ab_block_starts(const ab_obs *obs, double *out, long long n)
{
    double startr = obs->rlo;
    for (long long i = 0; i < n; i++, startr += obs->rstep) out[i] = startr;
}

void ab_preblock_starts(const ab_obs *obs, double *out, long long n)
{
    double startr = 8;
    for (long long i = 0; i < n; i++, startr += obs->rstep) out[i] = startr;
}

static int calc_fftlen(int numharm, int harmnum, int zmax, int wmax, const ab_obs *obs)
{                                                      /* src/accel_utils.c:137-150 */
    double f = (double) harmnum / (double) numharm;
    int bins_needed = (int) ceil(obs->corr_uselen * f) + 2;
    int end_effects = 2 * AB_NUMBETWEEN *
        ab_w_resp_halfwidth(ab_calc_required_z(f, zmax), ab_calc_required_w(f, wmax));
    return ab_next_good_fftlen(bins_needed + end_effects);
}

/* Correlation cost per template and transform (ms), by log2 L, as installed
 * by ab_set_transform_costs (ab_autotune measures it).  The initial table is
 * k_corr measured on a B200 (1965 MHz): 512 to 4096 points.  Lengths whose
 * entry is <= 0 are not used for superblocks; an all-zero table falls back
 * to the radix-16 work L log2 L for lengths up to 4096.  (8192-point
 * transforms run one 512-thread CTA per SM; in whole searches on B200 they
 * cost more than their calibrated figure, so the initial table leaves them
 * out.) */
static double g_costs[AB_COST_SLOTS] = {0, 0, 0, 0, 0, 0, 0, 0, 0,
                                        1.846e-6, 2.981e-6, 5.764e-6, 1.1243e-5, 0, 0, 0};
static pthread_mutex_t g_costs_mu = PTHREAD_MUTEX_INITIALIZER;

int ab_set_transform_costs(const double *costs, int n)
{
    if (n < 0 || (n > 0 && !costs)) return AB_ERR_ARG;
    pthread_mutex_lock(&g_costs_mu);
    for (int i = 0; i < AB_COST_SLOTS; i++) g_costs[i] = (i < n) ? costs[i] : 0.0;
    pthread_mutex_unlock(&g_costs_mu);
    return AB_OK;
}

int ab_get_transform_costs(double *costs, int n)
{
    if (!costs || n < 0) return AB_ERR_ARG;
    pthread_mutex_lock(&g_costs_mu);
    for (int i = 0; i < n; i++) costs[i] = (i < AB_COST_SLOTS) ? g_costs[i] : 0.0;
    pthread_mutex_unlock(&g_costs_mu);
    return AB_OK;
}

/* Cost of one transform of length L, or a negative value when L is not a
 * candidate (no measured entry). */
static double transform_cost(const double *cost_by_log2L, int L)
{
    int lg = twon_to_index(L);
    int any = 0;
    for (int i = 0; cost_by_log2L && i < AB_COST_SLOTS; i++) any |= cost_by_log2L[i] > 0.0;
    if (!any) return L <= 4096 ? (double) L * lg : -1.0;
    return (lg < AB_COST_SLOTS && cost_by_log2L[lg] > 0.0) ? cost_by_log2L[lg] : -1.0;
}

int ab_bankset_init(const ab_obs *obs, ab_bankset *bs)
{
    double c[AB_COST_SLOTS];
    ab_get_transform_costs(c, AB_COST_SLOTS);
    return ab_bankset_init_tuned(obs, c, bs);
}

int ab_bankset_init_tuned(const ab_obs *obs, const double *cost_by_log2L, ab_bankset *bs)
{
    memset(bs, 0, sizeof(*bs));
    int pairs[AB_MAX_BANKS][2], n = 0;
    pairs[n][0] = 1; pairs[n][1] = 1; n++;
    if (!obs->inmem)
        for (int s = 1; s < obs->numharmstages; s++)
            for (int h = 1; h < (1 << s); h += 2) {
                if (n >= AB_MAX_BANKS) return AB_ERR_ARG;
                pairs[n][0] = 1 << s; pairs[n][1] = h; n++;
            }
    long long nblocks = ab_num_blocks(obs), npre = ab_num_preblocks(obs);
    long long tmpl = 0, plane = 0, xhat = 0, dtime = 0;
    for (int i = 0; i < n; i++) {
        ab_bank *b = &bs->b[i];
        b->numharm = pairs[i][0];
        b->harmnum = pairs[i][1];
        b->stage = twon_to_index(b->numharm);
        b->f = (double) b->harmnum / (double) b->numharm;
        b->zmax = ab_calc_required_z(b->f, (int) obs->zhi);
        b->wmax = ab_calc_required_w(b->f, (int) obs->whi);
        b->nz = (b->zmax / AB_DZ) * 2 + 1;
        b->nw = (b->wmax / AB_DW) * 2 + 1;
        b->ntmpl = b->nz * b->nw;
        b->fftlen_ref = (i == 0) ? obs->fftlen
                      : calc_fftlen(b->numharm, b->harmnum, (int) obs->zhi, (int) obs->whi, obs);
        b->hw0 = ab_w_resp_halfwidth((double) -b->zmax, (double) -b->wmax);
        /* kern[0][0] has the widest response (src/accel_utils.c:1068-1071) */
        for (int wi = 0; wi < b->nw; wi++)
            for (int zi = 0; zi < b->nz; zi++)
                if (ab_w_resp_halfwidth(-b->zmax + zi * AB_DZ, -b->wmax + wi * AB_DW) > b->hw0)
                    return AB_ERR_ARG;
        int nrmax = 0;
        long long *rlo = (long long *) malloc(sizeof(long long) * (size_t) (nblocks > 0 ? nblocks : 1));
        int *nrs = (int *) malloc(sizeof(int) * (size_t) (nblocks > 0 ? nblocks : 1));
        if (!rlo || !nrs) {
            free(rlo);
            free(nrs);
            return AB_ERR_NOMEM;
        }
        double startr = obs->rlo;
        for (long long k = 0; k < nblocks; k++, startr += obs->rstep) {
            ab_hgeom g = ab_harm_geom(startr, startr + obs->rstep - AB_DR, b->numharm,
                                      b->harmnum, obs->zlo, obs->wlo, obs->corr_uselen);
            if (g.numrs > nrmax) nrmax = g.numrs;
            rlo[k] = g.rlo;
            nrs[k] = g.numrs;
        }
        if (npre > 0 && obs->corr_uselen > nrmax) nrmax = obs->corr_uselen;
        if (nrmax == 0) nrmax = obs->corr_uselen;
        b->numrs_max = nrmax;
        b->index = i;
        /* Valid cells read spread-data samples [0, 4*hw0 + numrs - 1).  The
         * device transforms the reference's window extended periodically
         * (period fftlen_ref), so any length >= that span gives the
         * reference's circular correlation on the valid cells, including
         * the cases where the reference's own FFT wraps into them. */
        int need = 4 * b->hw0 + nrmax - 1;
        int L = (int) next_pow2(need);
        if (L < 512) L = 512;
        if (L > 4096) {
            free(rlo);
            free(nrs);
            return AB_ERR_ARG;
        }
        /* Superblocks (standard search only): when the reference's own
         * transform does not wrap into valid cells, m consecutive blocks can
         * share one device transform of length L2 over the first block's
         * window, provided the widest span of m consecutive blocks'
         * sub-planes, 2 (rlo_last - rlo_first) + numrs_last columns, plus the
         * 4 hw0 - 1 samples of template reach fits in L2.  (L2, m) minimises
         * the transform cost per block. */
        int sbm = 1;
        double best = transform_cost(cost_by_log2L, L);
        /* not with the local-power normalisation: it scales every bin of
         * each block's own window, which one shared transform cannot hold */
        if (!obs->inmem && obs->norm_type == 0 && need <= b->fftlen_ref && nblocks > 1 &&
            best > 0.0) {
            for (int m = 2; m <= AB_MAX_SBM && m <= nblocks; m++) {
                long long span = 0;
                for (long long k = 0; k + m - 1 < nblocks; k++) {
                    long long sp = 2 * (rlo[k + m - 1] - rlo[k]) + nrs[k + m - 1];
                    if (sp > span) span = sp;
                }
                long long need_m = 4LL * b->hw0 + span - 1;
                /* 8192-point transforms only for w = 0 banks: their template
                 * generation holds the placed kernel (128 KiB) and no chirp
                 * in shared memory */
                const int lmax = b->wmax == 0 ? 8192 : 4096;
                for (int L2 = 512; L2 <= lmax; L2 <<= 1) {
                    if (need_m > L2 || L2 < need) continue;
                    double c = transform_cost(cost_by_log2L, L2) / m;
                    if (c > 0.0 && c < best * 0.98) {
                        best = c;
                        L = L2;
                        sbm = m;
                    }
                }
            }
        }
        free(rlo);
        free(nrs);
        b->sbm = sbm;
        b->L = L;
        b->log2L = twon_to_index(L);
        b->tmpl_off = tmpl;
        tmpl += (long long) b->ntmpl * L;
        b->xhat_off = xhat;
        xhat += L / 2;
        b->dtime_off = dtime;
        dtime += b->fftlen_ref / AB_NUMBETWEEN;
        b->plane_off = plane;
        plane += (long long) b->nw * b->nz * b->numrs_max;
    }
    bs->nbanks = n;
    bs->tmpl_total = tmpl;
    bs->plane_per_block = plane;
    bs->xhat_per_block = xhat;
    bs->dtime_per_block = dtime;
    return AB_OK;
}

/* ------------------------------------------------------------------ */
/* candidate list: insert_new_accelcand (src/accel_utils.c:387-469)    */
/* ------------------------------------------------------------------ */
/* The reference keeps an r-ordered singly linked list and walks it from
 * the head for every threshold crossing.  Here the list is an array: the
 * walk's stopping node ("first node with r >= rr, else the last node") is
 * found by a galloping binary search from the previous stop while the array
 * is ordered, and by the same linear walk as the reference while it is not
 * (replacing the second-to-last node with a higher r, or placing a new
 * candidate before a last node exactly 15 bins lower, can put two adjacent
 * nodes out of order).  ninv counts adjacent inversions exactly. */
struct ab_list {
    ab_cand *c;
    long long n, cap;
    long long ninv;                     /* adjacent pairs with r[i] > r[i+1] */
    long long last;                     /* stop node of the previous insert */
    double *seg;                        /* max-of-r segment tree (unordered walks) */
    long long segsz;
    int seg_dirty;
    /* the work-file lines of search_ffdotpows (src/accel_utils.c:1443-1447),
       one per candidate that an insertion adds, when wlog_on */
    int wlog_on;
    double wlog_T;
    char *wlog;
    size_t wlen, wcap;
    /* scratch of the batch replays (ab_replay_hits), kept for the list's
       next batch */
    void *scr;
    size_t scr_cap;
};

ab_list *ab_list_new(void)
{
    ab_list *l = (ab_list *) calloc(1, sizeof(ab_list));
    if (l) l->seg_dirty = 1;
    return l;
}

void ab_list_free(ab_list *l)
{
    if (!l) return;
    free(l->c);
    free(l->seg);
    free(l->wlog);
    free(l->scr);
    free(l);
}

void ab_list_worklog(ab_list *l, int on, double T)
{
    l->wlog_on = on;
    l->wlog_T = T;
}

const char *ab_list_worklog_text(const ab_list *l, size_t *len)
{
    *len = l->wlen;
    return l->wlog ? l->wlog : "";
}

static int wlog_line(ab_list *l, float power, float sigma, int numharm, double rr, double zz,
                     double ww)
{
    char b[2048];                   /* %f of doubles up to 1e308 fits */
    const int k = snprintf(b, sizeof b, "%-7.2f  %-7.4f  %-2d  %-14.4f  %-14.9f  %-10.4f %-10.4f\n",
                           power, sigma, numharm, rr, rr / l->wlog_T, zz, ww);
    if (k < 0 || (size_t) k >= sizeof b) return -1;
    if (l->wlen + (size_t) k + 1 > l->wcap) {
        size_t cap = l->wcap ? l->wcap : 4096;
        while (cap < l->wlen + (size_t) k + 1) cap *= 2;
        char *p = (char *) realloc(l->wlog, cap);
        if (!p) return -1;
        l->wlog = p;
        l->wcap = cap;
    }
    memcpy(l->wlog + l->wlen, b, (size_t) k + 1);
    l->wlen += (size_t) k;
    return 0;
}

/* Segment tree over the array positions holding max(r); answers "first
 * position in [0, lim) with r >= rr" in O(log n) whatever the ordering. */
static int seg_rebuild(ab_list *l)
{
    long long sz = 1;
    while (sz < l->n) sz <<= 1;
    if (sz != l->segsz || !l->seg) {
        double *p = (double *) realloc(l->seg, sizeof(double) * 2 * (size_t) sz);
        if (!p) return -1;
        l->seg = p;
        l->segsz = sz;
    }
    for (long long i = 0; i < sz; i++) l->seg[sz + i] = i < l->n ? l->c[i].r : -INFINITY;
    for (long long i = sz - 1; i >= 1; i--)
        l->seg[i] = l->seg[2 * i] > l->seg[2 * i + 1] ? l->seg[2 * i] : l->seg[2 * i + 1];
    l->seg_dirty = 0;
    return 0;
}

static void seg_set(ab_list *l, long long i)
{
    if (l->seg_dirty) return;
    long long pos = l->segsz + i;
    l->seg[pos] = l->c[i].r;
    for (pos >>= 1; pos >= 1; pos >>= 1)
        l->seg[pos] = l->seg[2 * pos] > l->seg[2 * pos + 1] ? l->seg[2 * pos] : l->seg[2 * pos + 1];
}

static long long seg_first_ge(const ab_list *l, long long node, long long lo, long long hi,
                              long long lim, double rr)
{
    if (lo >= lim || l->seg[node] < rr) return -1;
    if (hi - lo == 1) return lo;
    long long mid = (lo + hi) / 2;
    long long r = seg_first_ge(l, 2 * node, lo, mid, lim, rr);
    if (r >= 0) return r;
    return seg_first_ge(l, 2 * node + 1, mid, hi, lim, rr);
}

static int list_reserve(ab_list *l, long long want)
{
    if (want <= l->cap) return 0;
    long long nc = l->cap ? 2 * l->cap : 256;
    while (nc < want) nc *= 2;
    ab_cand *p = (ab_cand *) realloc(l->c, sizeof(ab_cand) * (size_t) nc);
    if (!p) return -1;
    l->c = p;
    l->cap = nc;
    return 0;
}

static void set_cand(ab_cand *c, float power, float sigma, int numharm, double rr,
                     double zz, double ww)
{
    c->power = power; c->sigma = sigma; c->numharm = numharm;
    c->r = rr; c->z = zz; c->w = ww;
}

static int inv_at(const ab_list *l, long long a)  /* pair (a, a+1) inverted? */
{
    return a >= 0 && a + 1 < l->n && l->c[a].r > l->c[a + 1].r;
}

static void replace_at(ab_list *l, long long i, float power, float sigma, int numharm,
                       double rr, double zz, double ww)
{
    l->ninv -= inv_at(l, i - 1) + inv_at(l, i);
    set_cand(&l->c[i], power, sigma, numharm, rr, zz, ww);
    l->ninv += inv_at(l, i - 1) + inv_at(l, i);
    seg_set(l, i);
}

static void insert_at(ab_list *l, long long at, float power, float sigma, int numharm,
                      double rr, double zz, double ww)
{
    l->ninv -= inv_at(l, at - 1);
    memmove(&l->c[at + 1], &l->c[at], sizeof(ab_cand) * (size_t) (l->n - at));
    set_cand(&l->c[at], power, sigma, numharm, rr, zz, ww);
    l->n++;
    l->ninv += inv_at(l, at - 1) + inv_at(l, at);
    l->seg_dirty = 1;
}

static void remove_at(ab_list *l, long long t)
{
    l->ninv -= inv_at(l, t - 1) + inv_at(l, t);
    memmove(&l->c[t], &l->c[t + 1], sizeof(ab_cand) * (size_t) (l->n - t - 1));
    l->n--;
    l->ninv += inv_at(l, t - 1);
    l->seg_dirty = 1;
}

/* first i in [0, n-1) with c[i].r >= rr, else n-1 (the reference's walk) */
static long long find_stop(ab_list *l, double rr)
{
    const ab_cand *c = l->c;
    const long long n1 = l->n - 1;
    if (n1 <= 0) return 0;
    if (l->ninv) {
        if (l->seg_dirty && seg_rebuild(l)) {        /* no memory: plain walk */
            long long t = 0;
            while (t < n1 && c[t].r < rr) t++;
            return t;
        }
        long long t = seg_first_ge(l, 1, 0, l->segsz, n1, rr);
        return t < 0 ? n1 : t;
    }
    long long s0 = l->last < 0 ? 0 : (l->last >= n1 ? n1 - 1 : l->last);
    long long lo, hi, step = 1;
    if (c[s0].r >= rr) {
        hi = s0;
        while (hi - step >= 0 && c[hi - step].r >= rr) { hi -= step; step <<= 1; }
        lo = hi - step < -1 ? -1 : hi - step;
    } else {
        lo = s0;
        while (lo + step < n1 && c[lo + step].r < rr) { lo += step; step <<= 1; }
        hi = lo + step > n1 ? n1 : lo + step;
    }
    while (hi - lo > 1) {
        long long mid = lo + (hi - lo) / 2;
        if (c[mid].r >= rr) hi = mid; else lo = mid;
    }
    l->last = hi;
    return hi;
}

int ab_list_insert(ab_list *l, float power, float sigma, int numharm,
                   double rr, double zz, double ww)
{
    if (list_reserve(l, l->n + 1)) return -1;
    if (l->n == 0) {
        set_cand(&l->c[0], power, sigma, numharm, rr, zz, ww);
        l->n = 1;
        if (l->wlog_on && wlog_line(l, power, sigma, numharm, rr, zz, ww)) return -1;
        return 1;
    }
    long long t = find_stop(l, rr);
    long long p = t - 1;
    ab_cand *c = l->c;
    int added = 0;
    double next_diff = fabs(rr - c[t].r);
    double prev_diff = p >= 0 ? fabs(rr - c[p].r) : AB_CLOSEST_R + 1.0;
    if (prev_diff < AB_CLOSEST_R) {
        if (c[p].sigma < sigma) {
            replace_at(l, p, power, sigma, numharm, rr, zz, ww);
            added = 1;
        }
        if (next_diff < AB_CLOSEST_R && c[t].sigma < sigma) {
            if (added) {              /* the new candidate already replaced prev */
                remove_at(l, t);
            } else {
                replace_at(l, t, power, sigma, numharm, rr, zz, ww);
                added = 1;
            }
        }
    } else if (next_diff < AB_CLOSEST_R) {
        if (c[t].sigma < sigma) {
            replace_at(l, t, power, sigma, numharm, rr, zz, ww);
            added = 1;
        }
    } else {
        added = 1;
        long long at = (t == l->n - 1 && c[t].r < rr - AB_CLOSEST_R) ? l->n : t;
        insert_at(l, at, power, sigma, numharm, rr, zz, ww);
    }
    if (added && l->wlog_on && wlog_line(l, power, sigma, numharm, rr, zz, ww)) return -1;
    return added;
}

long long ab_list_get(const ab_list *l, ab_cand *out, long long maxout)
{
    if (out)
        for (long long i = 0; i < l->n && i < maxout; i++) out[i] = l->c[i];
    return l->n;
}

/* Parallel LSD radix sort of hit indices by key.  Keys are taken relative
 * to the smallest present and sorted in equal digits of at most 14 bits (a
 * batch's re-packed keys need two or three passes), each pass a per-thread
 * histogram, an exclusive scan over (digit, thread) and a stable scatter. */
#define RS_MAXBITS 14                   /* digit width at most; 2^14 bins per thread */
#define RS_MAXT 16

typedef struct {
    const unsigned long long *k0;
    unsigned long long *k1;
    const unsigned long long *o0;       /* payload: power and sigma bits */
    unsigned long long *o1;
    size_t lo, hi;
    int shift;
    unsigned mask;
    size_t *hist;                       /* [nbins] of this thread */
} rs_job;

typedef struct {
    rs_job job[RS_MAXT];
    int nt, phase;
    pthread_barrier_t bar;
    size_t *hist;                       /* [nt][nbins] */
    int npasses, dbits;
    size_t nbins;
    unsigned long long *ka, *kb;
    unsigned long long *oa, *ob;
    size_t n;
} rs_ctx;

typedef struct { rs_ctx *c; int id; } rs_arg;

static void rs_count(rs_job *j)
{
    memset(j->hist, 0, sizeof(size_t) * ((size_t) j->mask + 1));
    for (size_t i = j->lo; i < j->hi; i++) j->hist[(j->k0[i] >> j->shift) & j->mask]++;
}

static void rs_scatter(rs_job *j)
{
    for (size_t i = j->lo; i < j->hi; i++) {
        size_t pos = j->hist[(j->k0[i] >> j->shift) & j->mask]++;
        j->k1[pos] = j->k0[i];
        j->o1[pos] = j->o0[i];
    }
}

static void rs_scan(rs_ctx *c)
{
    size_t sum = 0;
    for (size_t d = 0; d < c->nbins; d++)
        for (int t = 0; t < c->nt; t++) {
            size_t v = c->hist[(size_t) t * c->nbins + d];
            c->hist[(size_t) t * c->nbins + d] = sum;
            sum += v;
        }
}

static void rs_setup_pass(rs_ctx *c, int pass)
{
    unsigned long long *k0 = (pass & 1) ? c->kb : c->ka, *k1 = (pass & 1) ? c->ka : c->kb;
    unsigned long long *o0 = (pass & 1) ? c->ob : c->oa, *o1 = (pass & 1) ? c->oa : c->ob;
    for (int t = 0; t < c->nt; t++) {
        rs_job *j = &c->job[t];
        j->k0 = k0; j->k1 = k1; j->o0 = o0; j->o1 = o1;
        j->shift = c->dbits * pass;
        j->mask = (unsigned) (c->nbins - 1);
    }
}

static void *rs_worker(void *p)
{
    rs_arg *a = (rs_arg *) p;
    rs_ctx *c = a->c;
    for (int pass = 0; pass < c->npasses; pass++) {
        if (a->id == 0) rs_setup_pass(c, pass);
        pthread_barrier_wait(&c->bar);
        rs_count(&c->job[a->id]);
        pthread_barrier_wait(&c->bar);
        if (a->id == 0) rs_scan(c);
        pthread_barrier_wait(&c->bar);
        rs_scatter(&c->job[a->id]);
        pthread_barrier_wait(&c->bar);
    }
    return NULL;
}

static int g_active_sorts = 0;

/* Sorts keys[] (and the payload pl[] with it) in place by key; kb and ob
 * (n each) are work arrays, allocated here when NULL. */
static int radix_sort_kv(unsigned long long *keys, unsigned long long *pl, long long n,
                         unsigned long long *kb, unsigned long long *ob)
{
    unsigned long long kmin = ~0ull, kmax = 0;
    for (long long i = 0; i < n; i++) {
        if (keys[i] < kmin) kmin = keys[i];
        if (keys[i] > kmax) kmax = keys[i];
    }
    int bits = 0;
    while (bits < 64 && ((kmax - kmin) >> bits)) bits++;
    int npasses = (bits + RS_MAXBITS - 1) / RS_MAXBITS;
    if (npasses == 0) return AB_OK;
    const int dbits = (bits + npasses - 1) / npasses;     /* equal digits, at most 14 bits */
    rs_ctx c;
    memset(&c, 0, sizeof(c));
    /* sorts running at once (several contexts replaying, e.g. a request
     * pool's workers) share the host's cores */
    long ncpu = sysconf(_SC_NPROCESSORS_ONLN);
    const int active = __atomic_add_fetch(&g_active_sorts, 1, __ATOMIC_SEQ_CST);
    long share = (ncpu < 1 ? 1 : ncpu) / active;
    if (share < 1) share = 1;
    c.nt = n < (1 << 16) ? 1 : (int) (share > RS_MAXT ? RS_MAXT : share);
    c.n = (size_t) n;
    c.npasses = npasses;
    c.dbits = dbits;
    c.nbins = (size_t) 1 << dbits;
    c.ka = keys;
    c.oa = pl;
    const int own = !kb || !ob;
    c.kb = own ? (unsigned long long *) malloc(sizeof(unsigned long long) * (size_t) n) : kb;
    c.ob = own ? (unsigned long long *) malloc(sizeof(unsigned long long) * (size_t) n) : ob;
    c.hist = (size_t *) malloc(sizeof(size_t) * c.nbins * (size_t) c.nt);
    if (!c.kb || !c.ob || !c.hist) {
        if (own) { free(c.kb); free(c.ob); }
        free(c.hist);
        __atomic_sub_fetch(&g_active_sorts, 1, __ATOMIC_SEQ_CST);
        return AB_ERR_NOMEM;
    }
    for (long long i = 0; i < n; i++) keys[i] -= kmin;
    for (int t = 0; t < c.nt; t++) {
        c.job[t].lo = (size_t) n * t / c.nt;
        c.job[t].hi = (size_t) n * (t + 1) / c.nt;
        c.job[t].hist = c.hist + (size_t) t * c.nbins;
    }
    if (c.nt == 1) {
        for (int pass = 0; pass < npasses; pass++) {
            rs_setup_pass(&c, pass);
            rs_count(&c.job[0]);
            rs_scan(&c);
            rs_scatter(&c.job[0]);
        }
    } else {
        pthread_t th[RS_MAXT];
        rs_arg args[RS_MAXT];
        pthread_barrier_init(&c.bar, NULL, (unsigned) c.nt);
        for (int t = 1; t < c.nt; t++) {
            args[t].c = &c; args[t].id = t;
            pthread_create(&th[t], NULL, rs_worker, &args[t]);
        }
        args[0].c = &c; args[0].id = 0;
        rs_worker(&args[0]);
        for (int t = 1; t < c.nt; t++) pthread_join(th[t], NULL);
        pthread_barrier_destroy(&c.bar);
    }
    if (npasses & 1) {
        memcpy(keys, c.kb, sizeof(unsigned long long) * (size_t) n);
        memcpy(pl, c.ob, sizeof(unsigned long long) * (size_t) n);
    }
    for (long long i = 0; i < n; i++) keys[i] += kmin;
    if (own) { free(c.kb); free(c.ob); }
    free(c.hist);
    __atomic_sub_fetch(&g_active_sorts, 1, __ATOMIC_SEQ_CST);
    return AB_OK;
}

/* ------------------------------------------------------------------ */
/* exact parallel replay of one batch of threshold crossings            */
/* ------------------------------------------------------------------ */
/* An insertion at rr reads and changes only candidates closer than
 * AB_CLOSEST_R to rr, with two exceptions at the list's last node (the
 * reference's walk stops there whatever its r).  So the batch's crossings and
 * the list's candidates are cut into clusters: runs of occupied r bins 16
 * wide, which puts every two points of different clusters more than
 * AB_CLOSEST_R apart.  Each cluster replays its crossings, in the
 * batch's order, through ab_list_insert on a list of its own candidates.
 * While a higher cluster holds a candidate, the walk of this cluster's
 * insertions stops at that candidate rather than at this cluster's last one;
 * a sentinel node at r = +inf (never within AB_CLOSEST_R, never replaced)
 * stands for it from the first crossing of the batch after which it exists.
 * The clusters' lists are then concatenated in r order and the work-file
 * lines written in the batch's order. */
typedef struct {
    long long h0, nh;                   /* crossings: idx[h0 .. h0 + nh) */
    long long e0, ne;                   /* candidates: list positions [e0, e0 + ne) */
    long long tail_until;               /* first crossing index with a higher candidate */
    ab_list *out;
} rp_cluster;

typedef struct {
    const float *pw, *sg;
    const int *nh;
    const double *rr, *zz, *ww;
    const long long *idx;               /* crossings grouped by cluster, batch order within */
    unsigned char *added;
    const ab_cand *old;                 /* the list before the batch */
    rp_cluster *cl;
    const int *order;                   /* clusters, most crossings first */
    int ncl;
    int next;                           /* work counter */
    int err;
} rp_ctx;

static void *rp_worker(void *arg)
{
    rp_ctx *c = (rp_ctx *) arg;
    for (;;) {
        const int k = __atomic_fetch_add(&c->next, 1, __ATOMIC_SEQ_CST);
        if (k >= c->ncl) break;
        rp_cluster *q = &c->cl[c->order[k]];
        if (q->nh == 0) continue;            /* unchanged: its candidates are copied as they are */
        ab_list *l = ab_list_new();
        if (!l || list_reserve(l, q->ne + 2)) { __atomic_store_n(&c->err, 1, __ATOMIC_SEQ_CST); ab_list_free(l); continue; }
        for (long long i = 0; i < q->ne; i++) {
            l->c[i] = c->old[q->e0 + i];
            if (i > 0 && l->c[i - 1].r > l->c[i].r) l->ninv++;
        }
        l->n = q->ne;
        l->last = -1;
        int sentinel = 0;
        for (long long j = 0; j < q->nh; j++) {
            const long long h = c->idx[q->h0 + j];
            if (!sentinel && h >= q->tail_until) {
                if (list_reserve(l, l->n + 1)) { __atomic_store_n(&c->err, 1, __ATOMIC_SEQ_CST); break; }
                set_cand(&l->c[l->n], 0.0f, INFINITY, 0, INFINITY, 0.0, 0.0);
                l->n++;
                l->seg_dirty = 1;
                sentinel = 1;
            }
            const int a = ab_list_insert(l, c->pw[h], c->sg[h], c->nh[h], c->rr[h], c->zz[h], c->ww[h]);
            if (a < 0) { __atomic_store_n(&c->err, 1, __ATOMIC_SEQ_CST); break; }
            c->added[h] = (unsigned char) a;
        }
        if (sentinel) l->n--;                 /* the sentinel stays the last node */
        q->out = l;
    }
    return NULL;
}

/* Replays n crossings (power, sigma, harmonics, r, z, w in the reference's
 * visit order) into l exactly as n calls of ab_list_insert would, on up to
 * nthreads threads.  Returns AB_OK, or AB_ERR_ARG when the clusters cannot be
 * formed (the caller then replays serially), or AB_ERR_NOMEM. */
static int cmp_ll_desc(const void *a, const void *b)
{
    const long long x = *(const long long *) a, y = *(const long long *) b;
    return (x < y) - (x > y);
}

static int replay_clusters(ab_list *l, long long n, const float *pw, const float *sg,
                           const int *nh, const double *rr, const double *zz, const double *ww,
                           int nthreads, int *hcl, long long *idx, unsigned char *added)
{
    if (n <= 0) return AB_OK;
    /* bins of width AB_CLOSEST_R over every point */
    double rmax = 0.0;
    for (long long i = 0; i < n; i++) {
        if (!(rr[i] >= 0.0) || rr[i] > 1e12) return AB_ERR_ARG;
        if (rr[i] > rmax) rmax = rr[i];
    }
    for (long long i = 0; i < l->n; i++) {
        if (!(l->c[i].r >= 0.0) || l->c[i].r > 1e12) return AB_ERR_ARG;
        if (l->c[i].r > rmax) rmax = l->c[i].r;
    }
    /* bins 16 bins wide (>= AB_CLOSEST_R; r * 1/16 is exact) */
    const long long nb = (long long) (rmax * 0.0625) + 2;
    if (nb > (1LL << 31)) return AB_ERR_ARG;
    int *bin = (int *) calloc((size_t) nb, sizeof(int));          /* occupied, then cluster + 1 */
    if (!bin) return AB_ERR_NOMEM;
    memset(added, 0, (size_t) n);
    for (long long i = 0; i < n; i++) {
        hcl[i] = (int) (rr[i] * 0.0625);
        bin[hcl[i]] = 1;
    }
    for (long long i = 0; i < l->n; i++) bin[(long long) (l->c[i].r * 0.0625)] = 1;
    int ncl = 0;
    for (long long b = 0; b < nb; b++)
        if (bin[b]) bin[b] = (b > 0 && bin[b - 1]) ? bin[b - 1] : ++ncl;
    if (ncl >= (1 << 24)) { free(bin); return AB_ERR_ARG; }
    rp_cluster *cl = (rp_cluster *) calloc((size_t) ncl, sizeof(rp_cluster));
    int *order = (int *) malloc(sizeof(int) * (size_t) ncl);
    int rc = AB_OK;
    if (!cl || !order) { rc = AB_ERR_NOMEM; goto done; }
    /* crossings grouped by cluster, each group in batch order */
    for (long long i = 0; i < n; i++) {
        hcl[i] = bin[hcl[i]] - 1;
        cl[hcl[i]].nh++;
    }
    {
        long long s = 0;
        for (int k = 0; k < ncl; k++) { cl[k].h0 = s; s += cl[k].nh; cl[k].nh = 0; }
    }
    for (long long i = 0; i < n; i++) {
        rp_cluster *q = &cl[hcl[i]];
        idx[q->h0 + q->nh++] = i;
    }
    /* each cluster's candidates must be one run of list positions, in cluster order */
    for (int k = 0; k < ncl; k++) cl[k].e0 = -1;
    {
        int prev = -1;
        for (long long i = 0; i < l->n; i++) {
            const int k = bin[(long long) (l->c[i].r * 0.0625)] - 1;
            if (k < prev) { rc = AB_ERR_ARG; goto done; }
            if (k != prev) {
                if (cl[k].e0 >= 0) { rc = AB_ERR_ARG; goto done; }
                cl[k].e0 = i;
            }
            cl[k].ne++;
            prev = k;
        }
    }
    for (int k = 0; k < ncl; k++) if (cl[k].e0 < 0) cl[k].e0 = 0;
    /* the first crossing after which a higher cluster holds a candidate */
    {
        long long t = LLONG_MAX;
        for (int k = ncl - 1; k >= 0; k--) {
            cl[k].tail_until = t;
            const long long own = cl[k].ne > 0 ? -1 : (cl[k].nh > 0 ? idx[cl[k].h0] : LLONG_MAX);
            if (own < t) t = own;
        }
    }
    /* largest clusters first */
    {
        long long *ord = (long long *) malloc(sizeof(long long) * (size_t) ncl);
        if (!ord) { rc = AB_ERR_NOMEM; goto done; }
        for (int k = 0; k < ncl; k++) ord[k] = (cl[k].nh << 24) | (long long) ((1 << 24) - 1 - k);
        qsort(ord, (size_t) ncl, sizeof(long long), cmp_ll_desc);
        for (int k = 0; k < ncl; k++) order[k] = (1 << 24) - 1 - (int) (ord[k] & ((1 << 24) - 1));
        free(ord);
    }
    {
        rp_ctx c = {pw, sg, nh, rr, zz, ww, idx, added, l->c, cl, order, ncl, 0, 0};
        int nt = nthreads < 1 ? 1 : nthreads;
        if (nt > ncl) nt = ncl;
        if (nt > RS_MAXT) nt = RS_MAXT;
        pthread_t th[RS_MAXT];
        int started = 1;
        for (int t = 1; t < nt; t++)
            if (pthread_create(&th[t], NULL, rp_worker, &c) == 0) started++;
            else break;
        rp_worker(&c);
        for (int t = 1; t < started; t++) pthread_join(th[t], NULL);
        if (c.err) { rc = AB_ERR_NOMEM; goto done; }
    }
    /* concatenate the clusters' lists (or their unchanged candidates) in r order */
    {
        long long total = 0;
        for (int k = 0; k < ncl; k++) total += cl[k].out ? cl[k].out->n : cl[k].ne;
        long long cap = total > 256 ? total : 256;
        ab_cand *nc = (ab_cand *) malloc(sizeof(ab_cand) * (size_t) cap);
        if (!nc) { rc = AB_ERR_NOMEM; goto done; }
        long long pos = 0;
        for (int k = 0; k < ncl; k++) {
            ab_list *o = cl[k].out;
            const ab_cand *src = o ? o->c : l->c + cl[k].e0;
            const long long m = o ? o->n : cl[k].ne;
            if (m) memcpy(&nc[pos], src, sizeof(ab_cand) * (size_t) m);
            pos += m;
        }
        free(l->c);
        l->c = nc;
        l->cap = cap;
        l->n = total;
        l->ninv = 0;
        for (long long i = 0; i + 1 < l->n; i++) l->ninv += l->c[i].r > l->c[i + 1].r;
        l->last = -1;
        l->seg_dirty = 1;
    }
    if (l->wlog_on)
        for (long long i = 0; i < n; i++)
            if (added[i] && wlog_line(l, pw[i], sg[i], nh[i], rr[i], zz[i], ww[i])) {
                rc = AB_ERR_NOMEM;
                goto done;
            }
done:
    if (cl)
        for (int k = 0; k < ncl; k++) ab_list_free(cl[k].out);
    free(cl); free(order); free(bin);
    return rc;
}

int ab_list_replay_parallel(ab_list *l, long long n, const float *pw, const float *sg,
                            const int *nh, const double *rr, const double *zz, const double *ww,
                            int nthreads)
{
    if (n <= 0) return AB_OK;
    int *hcl = (int *) malloc(sizeof(int) * (size_t) n);
    long long *idx = (long long *) malloc(sizeof(long long) * (size_t) n);
    unsigned char *added = (unsigned char *) malloc((size_t) n);
    int rc = (hcl && idx && added)
                 ? replay_clusters(l, n, pw, sg, nh, rr, zz, ww, nthreads, hcl, idx, added)
                 : AB_ERR_NOMEM;
    free(hcl); free(idx); free(added);
    return rc;
}

/* Runs fn on nt jobs (job t at base + t * size), job 0 on this thread and
 * the others on threads of their own (on this one when a thread cannot be
 * started). */
static void run_jobs(void *(*fn)(void *), void *base, size_t size, int nt)
{
    pthread_t th[RS_MAXT];
    int ok[RS_MAXT] = {0};
    for (int t = 1; t < nt; t++)
        ok[t] = pthread_create(&th[t], NULL, fn, (char *) base + (size_t) t * size) == 0;
    fn(base);
    for (int t = 1; t < nt; t++) {
        if (ok[t]) pthread_join(th[t], NULL);
        else fn((char *) base + (size_t) t * size);
    }
}

/* Packing of crossings [lo, hi): power and sigma bits into one word, the
 * keys' used field bits and block range (pk_scan), then the keys re-packed
 * in those widths (pk_pack). */
typedef struct {
    unsigned long long *keys;
    const float *pows, *sigs;
    unsigned long long *pl;
    long long lo, hi;
    unsigned long long low, bmin, bmax;
    int wr, wz, ww, ws;
} pk_job;

static void *pk_scan(void *p)
{
    pk_job *j = (pk_job *) p;
    const int bsh = AB_KEY_RBITS + AB_KEY_ZBITS + AB_KEY_WBITS + AB_KEY_SBITS;
    unsigned long long low = 0, bmin = ~0ull, bmax = 0;
    for (long long i = j->lo; i < j->hi; i++) {
        unsigned pb, sb = 0;
        memcpy(&pb, &j->pows[i], 4);
        if (j->sigs) memcpy(&sb, &j->sigs[i], 4);
        j->pl[i] = ((unsigned long long) pb << 32) | sb;
        const unsigned long long k = j->keys[i], b = k >> bsh;
        low |= k & ((1ull << bsh) - 1);
        if (b < bmin) bmin = b;
        if (b > bmax) bmax = b;
    }
    j->low = low; j->bmin = bmin; j->bmax = bmax;
    return NULL;
}

static void *pk_pack(void *p)
{
    pk_job *j = (pk_job *) p;
    for (long long i = j->lo; i < j->hi; i++) {
        const unsigned long long k = j->keys[i];
        const unsigned long long r = k & 0xFFFF, z = (k >> AB_KEY_RBITS) & 0xFFF,
                                 w = (k >> (AB_KEY_RBITS + AB_KEY_ZBITS)) & 0x7F,
                                 st = (k >> (AB_KEY_RBITS + AB_KEY_ZBITS + AB_KEY_WBITS)) & 0x7,
                                 b = k >> (AB_KEY_RBITS + AB_KEY_ZBITS + AB_KEY_WBITS + AB_KEY_SBITS);
        j->keys[i] = (((((((b - j->bmin) << j->ws) | st) << j->ww | w) << j->wz) | z) << j->wr) | r;
    }
    return NULL;
}

/* The candidate fields of crossings [lo, hi) of a sorted batch (threads
 * share the loop; each keeps its own block geometry). */
typedef struct {
    const ab_obs *obs;
    unsigned long long *keys;           /* in: compact keys; out: the search's keys */
    const unsigned long long *pl;
    int wr, wz, ww, ws;                 /* field widths of the compact keys */
    unsigned long long bmin;
    float *pows, *sigs;                 /* out: the sorted powers (and sigmas) */
    const double *startr_tab;
    long long ntab, lo, hi;
    float *fsg; int *fnh; double *frr, *fzz, *fww;
    int err;
} rf_job;

static void *rf_worker(void *p)
{
    rf_job *j = (rf_job *) p;
    /* 1 / 2^stage is exact, so the products equal the reference's quotients */
    static const double inv[8] = {1.0, 0.5, 0.25, 0.125, 0.0625, 0.03125, 0.015625, 0.0078125};
    long long cur_block = -1;
    ab_hgeom g = {0, 0, 0, 0};
    for (long long i = j->lo; i < j->hi; i++) {
        unsigned long long k = j->keys[i];
        unsigned pb = (unsigned) (j->pl[i] >> 32), sb = (unsigned) j->pl[i];
        float pw, sg;
        memcpy(&pw, &pb, 4);
        memcpy(&sg, &sb, 4);
        j->pows[i] = pw;
        if (j->sigs) j->sigs[i] = sg;
        const int ri = (int) (k & ((1ull << j->wr) - 1)); k >>= j->wr;
        const int zi = (int) (k & ((1ull << j->wz) - 1)); k >>= j->wz;
        const int wi = (int) (k & ((1ull << j->ww) - 1)); k >>= j->ww;
        const int stage = (int) (k & ((1ull << j->ws) - 1)); k >>= j->ws;
        const long long block = (long long) (k + j->bmin);
        j->keys[i] = ((unsigned long long) block << (AB_KEY_RBITS + AB_KEY_ZBITS + AB_KEY_WBITS + AB_KEY_SBITS)) |
                     ((unsigned long long) stage << (AB_KEY_RBITS + AB_KEY_ZBITS + AB_KEY_WBITS)) |
                     ((unsigned long long) wi << (AB_KEY_RBITS + AB_KEY_ZBITS)) |
                     ((unsigned long long) zi << AB_KEY_RBITS) | (unsigned long long) ri;
        if (block >= j->ntab || stage > 7) { j->err = 1; return NULL; }
        if (block != cur_block) {
            /* the fundamental plane of the block (src/accel_utils.c:1034-1039) */
            double startr = j->startr_tab[block];
            g = ab_harm_geom(startr, startr + j->obs->rstep - AB_DR, 1, 1, j->obs->zlo,
                             j->obs->wlo, j->obs->corr_uselen);
            cur_block = block;
        }
        const int numharm = 1 << stage;
        j->fsg[i] = j->sigs ? sg
                            : (float) ab_candidate_sigma(pw, numharm,
                                                         (double) j->obs->numindep[stage]);
        j->fnh[i] = numharm;
        j->frr[i] = (g.rlo + ri * (double) AB_DR) * inv[stage];
        j->fzz[i] = (g.zlo + zi * (double) AB_DZ) * inv[stage];
        j->fww[i] = (g.wlo + wi * (double) AB_DW) * inv[stage];
    }
    return NULL;
}

/* Device hits carry (key, power, sigma); the key orders them as the
 * reference visits them (block, stage, w, z, r).  Sorts them (keys, pows and
 * sigs are reordered in place) and replays search_ffdotpows' per-hit work
 * (src/accel_utils.c:1430-1442).  sigs may be NULL, in which case
 * candidate_sigma is evaluated here.  Batches of AB_REPLAY_PARALLEL_MIN
 * crossings or more fill their candidate fields and replay on several threads
 * (ab_list_replay_parallel), into scratch the list keeps for its next batch. */
int ab_replay_hits(const ab_obs *obs, unsigned long long *keys, float *pows, float *sigs,
                   long long nhits, const double *startr_tab, long long ntab, ab_list *l)
{
    if (nhits <= 0) return AB_OK;
    const size_t n = (size_t) nhits;
    /* pl, kb, ob (8 B), fsg, fnh, hcl (4 B), frr, fzz, fww (8 B), idx (8 B), added (1 B) */
    const size_t need = n * (8 * 3 + 4 * 3 + 8 * 3 + 8 + 1) + 64;
    if (need > l->scr_cap) {
        /* 2 MiB-aligned and marked for huge pages: a batch of millions of
           crossings touches hundreds of MB once, and 4 KiB page faults on it
           would cost more than the replay */
        void *p = NULL;
        const size_t cap = (need + ((size_t) 2 << 20) - 1) & ~(((size_t) 2 << 20) - 1);
        if (posix_memalign(&p, (size_t) 2 << 20, cap)) return AB_ERR_NOMEM;
#ifdef MADV_HUGEPAGE
        madvise(p, cap, MADV_HUGEPAGE);
#endif
        free(l->scr);
        l->scr = p;
        l->scr_cap = cap;
    }
    unsigned long long *pl = (unsigned long long *) l->scr;
    unsigned long long *kb = pl + n, *ob = kb + n;
    double *frr = (double *) (ob + n), *fzz = frr + n, *fww = fzz + n;
    long long *idx = (long long *) (fww + n);
    float *fsg = (float *) (idx + n);
    int *fnh = (int *) (fsg + n), *hcl = fnh + n;
    unsigned char *added = (unsigned char *) (hcl + n);
    long ncpu = sysconf(_SC_NPROCESSORS_ONLN);
    const int active = __atomic_add_fetch(&g_active_sorts, 1, __ATOMIC_SEQ_CST);
    long share = (ncpu < 1 ? 1 : ncpu) / active;
    __atomic_sub_fetch(&g_active_sorts, 1, __ATOMIC_SEQ_CST);
    if (share < 1) share = 1;
    const int big = nhits >= AB_REPLAY_PARALLEL_MIN;
    int nt = big ? (int) (share > RS_MAXT ? RS_MAXT : share) : 1;
    /* the keys re-packed in the field widths this batch uses (the same
       order, fewer radix passes) */
    pk_job pk[RS_MAXT];
    for (int t = 0; t < nt; t++) {
        pk_job j = {keys, pows, sigs, pl, nhits * t / nt, nhits * (t + 1) / nt, 0, ~0ull, 0,
                    0, 0, 0, 0};
        pk[t] = j;
    }
    run_jobs(pk_scan, pk, sizeof(pk_job), nt);
    unsigned long long low = 0, bmin = ~0ull, bmax = 0;
    for (int t = 0; t < nt; t++) {
        low |= pk[t].low;
        if (pk[t].bmin < bmin) bmin = pk[t].bmin;
        if (pk[t].bmax > bmax) bmax = pk[t].bmax;
    }
    int wr = 0, wz = 0, ww = 0, ws = 0;
    while (wr < 16 && ((low & 0xFFFF) >> wr)) wr++;
    while (wz < 12 && (((low >> AB_KEY_RBITS) & 0xFFF) >> wz)) wz++;
    while (ww < 7 && (((low >> (AB_KEY_RBITS + AB_KEY_ZBITS)) & 0x7F) >> ww)) ww++;
    while (ws < 3 && (((low >> (AB_KEY_RBITS + AB_KEY_ZBITS + AB_KEY_WBITS)) & 0x7) >> ws)) ws++;
    for (int t = 0; t < nt; t++) {
        pk[t].bmin = bmin;
        pk[t].wr = wr; pk[t].wz = wz; pk[t].ww = ww; pk[t].ws = ws;
    }
    run_jobs(pk_pack, pk, sizeof(pk_job), nt);
    (void) bmax;
    int rc = radix_sort_kv(keys, pl, nhits, kb, ob);
    if (rc) return rc;
    rf_job jobs[RS_MAXT];
    for (int t = 0; t < nt; t++) {
        rf_job j = {obs, keys, pl, wr, wz, ww, ws, bmin, pows, sigs, startr_tab, ntab,
                    nhits * t / nt, nhits * (t + 1) / nt, fsg, fnh, frr, fzz, fww, 0};
        jobs[t] = j;
    }
    run_jobs(rf_worker, jobs, sizeof(rf_job), nt);
    for (int t = 0; t < nt; t++)
        if (jobs[t].err) return AB_ERR_ARG;
    if (big) {
        rc = replay_clusters(l, nhits, pows, fsg, fnh, frr, fzz, fww, (int) share, hcl, idx,
                             added);
        if (rc != AB_ERR_ARG) return rc;
    }
    /* small batches, or crossings that cannot be cut into clusters */
    for (long long i = 0; i < nhits; i++)
        if (ab_list_insert(l, pows[i], fsg[i], fnh[i], frr[i], fzz[i], fww[i]) < 0)
            return AB_ERR_NOMEM;
    return AB_OK;
}

/* ------------------------------------------------------------------ */
/* post-search list handling                                            */
/* ------------------------------------------------------------------ */

/* sort_accelcands: stable sort by decreasing sigma, ties by decreasing
 * power (src/accel_utils.c:364-384; g_slist_sort is a stable merge sort). */
static int cand_before(const ab_cand *a, const ab_cand *b)
{
    int r = (a->sigma < b->sigma) - (a->sigma > b->sigma);
    if (!r) r = (a->power < b->power) - (a->power > b->power);
    return r;
}

int ab_sort_cands(ab_cand *c, long long n)
{
    if (n < 2) return AB_OK;
    ab_cand *tmp = (ab_cand *) malloc(sizeof(ab_cand) * (size_t) n);
    if (!tmp) return AB_ERR_NOMEM;
    for (long long w = 1; w < n; w *= 2) {                 /* bottom-up merge sort */
        for (long long lo = 0; lo < n; lo += 2 * w) {
            long long mid = lo + w < n ? lo + w : n, hi = lo + 2 * w < n ? lo + 2 * w : n;
            long long i = lo, j = mid, k = lo;
            while (i < mid && j < hi) tmp[k++] = (cand_before(&c[j], &c[i]) < 0) ? c[j++] : c[i++];
            while (i < mid) tmp[k++] = c[i++];
            while (j < hi) tmp[k++] = c[j++];
        }
        memcpy(c, tmp, sizeof(ab_cand) * (size_t) n);
    }
    free(tmp);
    return AB_OK;
}

/* eliminate_harmonics (src/accel_utils.c:472-549) on a sorted array. */
long long ab_eliminate_harmonics(ab_cand *c, long long n)
{
    static const double ratios[23][2] = {
        {3, 2}, {5, 2}, {2, 3}, {4, 3}, {5, 3}, {3, 4}, {5, 4}, {2, 5}, {3, 5}, {4, 5},
        {5, 6}, {2, 7}, {3, 7}, {4, 7}, {3, 8}, {5, 8}, {2, 9}, {3, 10}, {2, 11},
        {3, 11}, {2, 13}, {3, 13}, {2, 15}};
    const int maxharm = 16;
    const double tooclose = 1.5;
    char *gone = (char *) calloc((size_t) (n > 0 ? n : 1), 1);
    long long cur = 0;
    for (;;) {
        long long nx = cur + 1;
        while (nx < n && gone[nx]) nx++;
        if (nx >= n) break;
        for (long long o = nx; o < n; o++) {
            if (gone[o]) continue;
            int remove = 0;
            for (int ii = 1; ii <= maxharm && !remove; ii++)
                if (fabs(c[cur].r / ii - c[o].r) < tooclose) remove = 1;
            for (int ii = 1; ii <= maxharm && !remove; ii++)
                if (fabs(c[cur].r * ii - c[o].r) < tooclose) remove = 1;
            for (int k = 0; k < 23 && !remove; k++)
                if (fabs(c[cur].r * ratios[k][0] / ratios[k][1] - c[o].r) < tooclose) remove = 1;
            if (remove) gone[o] = 1;
        }
        cur = nx;
        while (cur < n && gone[cur]) cur++;
        if (cur >= n) break;
    }
    long long m = 0;
    for (long long i = 0; i < n; i++)
        if (!gone[i]) c[m++] = c[i];
    free(gone);
    return m;
}

int ab_bank_geometry(const ab_obs *obs, int *nbanks, int *info, int maxbanks)
{
    ab_bankset bs;
    if (!obs || !nbanks) return AB_ERR_ARG;
    int rc = ab_bankset_init(obs, &bs);
    if (rc) return rc;
    *nbanks = bs.nbanks;
    if (!info) return AB_OK;
    if (maxbanks < bs.nbanks) return AB_ERR_OVERFLOW;
    for (int k = 0; k < bs.nbanks; k++) {
        const ab_bank *b = &bs.b[k];
        int *o = info + 9 * k;
        o[0] = b->numharm; o[1] = b->harmnum; o[2] = b->nz; o[3] = b->nw;
        o[4] = b->fftlen_ref; o[5] = b->L; o[6] = b->hw0; o[7] = b->numrs_max;
        o[8] = b->sbm;
    }
    return AB_OK;
}

/* copy_ffdotpows (src/accel_utils.c:1200-1217) into caller-owned storage. */
int ab_copy_ffdotpows(const ab_ffdotpows *src, ab_ffdotpows *dst)
{
    if (!src || !dst || (!src->powers && src->numrs > 0)) return AB_ERR_ARG;
    size_t n = (size_t) src->numws * src->numzs * src->numrs;
    if (!dst->powers || dst->capacity < n) return AB_ERR_OVERFLOW;
    dst->rlo = src->rlo;
    dst->zlo = src->zlo;
    dst->wlo = src->wlo;
    dst->numrs = src->numrs;
    dst->numzs = src->numzs;
    dst->numws = src->numws;
    if (n) memcpy(dst->powers, src->powers, sizeof(float) * n);
    return AB_OK;
}

/* get_fourier_amplitudes (src/accel_utils.c:993-1022): the window
 * [lobin, lobin + numbins) of a spectrum that starts at bin obs->lobin, with
 * zeros where it runs off either end. */
int ab_get_fourier_amplitudes(const ab_obs *obs, const ab_fcomplex *fft, long long lobin,
                              int numbins, ab_fcomplex *out)
{
    if (!obs || !fft || !out || numbins < 0) return AB_ERR_ARG;
    for (int i = 0; i < numbins; i++) {
        long long b = lobin - obs->lobin + i;
        if (b >= 0 && b < obs->numbins) out[i] = fft[b];
        else out[i].r = out[i].i = 0.0f;
    }
    return AB_OK;
}

/* The block partition of deredden (src/misc_utils.c:912-1038): after bin 0,
 * a first block of startwidth bins, then blocks of startwidth ln(binnum)
 * bins (capped at endwidth, and endwidth once binnum / T reaches endfreq),
 * the last one cut at the end of the spectrum.  blocks[2k] = first bin,
 * blocks[2k+1] = length.  Returns AB_ERR_ARG when the spectrum is shorter
 * than the first block, AB_ERR_OVERFLOW past maxblocks. */
int ab_dered_plan(long long numbins, int startwidth, int endwidth, double endfreq, double T,
                  int *blocks, long long maxblocks, long long *nblocks)
{
    if (!nblocks || startwidth < 1 || endwidth < startwidth || numbins < 1 + startwidth)
        return AB_ERR_ARG;
    const float Tf = (float) T;
    long long rpos = 1, binnum = 1, nb = 0;
    int bufflen = startwidth;
    for (;;) {
        long long n = numbins - rpos < bufflen ? numbins - rpos : bufflen;
        if (n <= 0) break;
        if (blocks) {
            if (nb >= maxblocks) return AB_ERR_OVERFLOW;
            blocks[2 * nb] = (int) rpos;
            blocks[2 * nb + 1] = (int) n;
        }
        nb++;
        rpos += n;
        binnum += n;
        if (nb == 1 || (float) binnum / Tf < endfreq) {
            bufflen = (int) (startwidth * log((double) binnum));
            if (bufflen > endwidth) bufflen = endwidth;
        } else {
            bufflen = endwidth;
        }
    }
    *nblocks = nb;
    return AB_OK;
}

long long ab_num_blocks_main(const ab_obs *obs) { return obs ? ab_num_blocks(obs) : -1; }

/* ------------------------------------------------------------------ */
/* candidate properties and the .cand file                             */
/* ------------------------------------------------------------------ */

/* calc_props (src/characteristics.c:195-264): purity from the curvature of
 * the locally normalised power, then the errors of r, z, w, power, phase
 * and centroid.  The purity is stored as float first and the later
 * formulas use that stored value, as the reference's do. */
int ab_calc_props(const ab_rderivs *d, double r, double z, double w, ab_fourierprops *o)
{
    if (!d || !o) return AB_ERR_ARG;
    if (fabs(d->pow) < AB_DBLCORRECT || d->locpow < AB_DBLCORRECT) return AB_ERR_ARG;
    const double tmppow = d->pow / d->locpow, tmpd2pow = d->d2pow / d->locpow;
    memset(o, 0, sizeof *o);
    o->pur = (float) (sqrt(1.5 * fabs(tmpd2pow) / tmppow) / AB_PI);
    if (fabs(tmppow) < AB_DBLCORRECT) o->pur = 1.0f;
    o->purerr = (float) (1.0 / (o->pur * sqrt(10.0 * tmppow)));
    o->r = r;
    o->rerr = (float) (3.0 / (AB_PI * o->pur * sqrt(6.0 * tmppow)));
    o->z = z;
    o->zerr = (float) (3.0 * sqrt(10.0) / (AB_PI * o->pur * o->pur * sqrt(tmppow)));
    o->w = w;
    o->werr = (float) (6.0 * sqrt(105.0) / (AB_PI * o->pur * o->pur * o->pur * sqrt(tmppow)));
    o->pow = (float) tmppow;
    o->powerr = (float) sqrt(2.0 * tmppow);
    o->sig = (float) sqrt(2.0 * tmppow - log(AB_PI * tmppow));
    o->rawpow = (float) d->pow;
    o->phs = (float) d->phs;
    o->phserr = (float) (1.0 / o->powerr);
    o->cen = (float) (-d->dphs / (2.0 * AB_PI));
    o->cenerr = (float) (1.0 / sqrt(24.0 * tmppow));
    o->locpow = (float) d->locpow;
    return AB_OK;
}

/* calc_rzwerrs (src/characteristics.c:353-392): period, frequency, their
 * first two derivatives at the start of the run, and their errors. */
int ab_calc_rzwerrs(const ab_fourierprops *p, double T, ab_rzwerrs *o)
{
    if (!p || !o || !(T > 0.0)) return AB_ERR_ARG;
    const double T2 = T * T, T3 = T2 * T;
    /* the float errors are squared in float, as the reference does */
    const double r2 = p->r * p->r, sr2 = p->rerr * p->rerr, r4 = r2 * r2;
    const double z2 = p->z * p->z, sz2 = p->zerr * p->zerr;
    const double tmp = p->r * p->w - 3 * z2;
    memset(o, 0, sizeof *o);
    o->f = p->r / T;
    o->ferr = (float) (p->rerr / T);
    o->fd = p->z / T2;
    o->fderr = (float) (p->zerr / T2);
    o->fdd = p->w / T3;
    o->fdderr = (float) (p->werr / T3);
    o->p = T / p->r;
    o->perr = (float) (T * p->rerr / r2);
    o->pd = -p->z / r2;
    o->pderr = (float) sqrt(4 * z2 * sr2 / (r4 * r2) + sz2 / r4);
    o->pdd = p->w == 0.0 ? 0.0 : (2 * z2 - p->r * p->w) / (T * r2 * p->r);
    o->pdderr = (float) sqrt((p->werr * p->werr * r4 + 16 * sz2 * r2 + 4 * tmp * tmp * sr2) /
                             (r4 * r4 * T2));
    return AB_OK;
}

/* src/accelsearch.c:261-272: the fundamentals' properties written to the
 * .cand file. */
int ab_cand_props(const ab_cand *c, const ab_polished *pol, long long n, ab_fourierprops *out)
{
    if (n < 0 || (n > 0 && (!c || !pol || !out))) return AB_ERR_ARG;
    for (long long i = 0; i < n; i++) {
        if (c[i].numharm < 1) return AB_ERR_ARG;
        int rc = ab_calc_props(&pol[i].derivs[0], c[i].r, c[i].z, c[i].w, &out[i]);
        if (rc) return rc;
        out[i].rerr = (float) AB_DR / c[i].numharm;
        out[i].zerr = (float) AB_DZ / c[i].numharm;
        out[i].werr = (float) AB_DW / c[i].numharm;
    }
    return AB_OK;
}
