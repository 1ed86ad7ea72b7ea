/*
 * ab_host.c -- host C side of the engine: search geometry and thresholds
 * (create_accelobs), template-bank geometry (create_subharminfos),
 * statistics (candidate_sigma / power_for_sigma), and the candidate list
 * with the replay of device threshold crossings in reference order.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

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
    obs->norm_type = 0;
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

int ab_bankset_init(const ab_obs *obs, ab_bankset *bs)
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
    long long tmpl = 0, plane = 0, xhat = 0;
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
        double startr = obs->rlo;
        for (long long k = 0; k < nblocks; k++, startr += obs->rstep) {
            ab_hgeom g = ab_harm_geom(startr, startr + obs->rstep - AB_DR, b->numharm,
                                      b->harmnum, obs->zlo, obs->wlo, obs->corr_uselen);
            if (g.numrs > nrmax) nrmax = g.numrs;
        }
        if (npre > 0 && obs->corr_uselen > nrmax) nrmax = obs->corr_uselen;
        if (nrmax == 0) nrmax = obs->corr_uselen;
        b->numrs_max = nrmax;
        /* Valid cells use spread-data samples [0, 4*hw0 + numrs - 1); the
         * reference's circular FFT of fftlen_ref must not wrap into them,
         * which makes any transform length >= that span equivalent. */
        int need = 4 * b->hw0 + nrmax - 1;
        if (need > b->fftlen_ref) return AB_ERR_ARG;
        int L = (int) next_pow2(need);
        if (L < 512) L = 512;
        if (L > 4096) return AB_ERR_ARG;
        b->L = L;
        b->log2L = twon_to_index(L);
        b->tmpl_off = tmpl;
        tmpl += (long long) b->ntmpl * L;
        b->xhat_off = xhat;
        xhat += L / 2;
        b->plane_off = plane;
        plane += (long long) b->nw * b->nz * b->numrs_max;
    }
    bs->nbanks = n;
    bs->tmpl_total = tmpl;
    bs->plane_per_block = plane;
    bs->xhat_per_block = xhat;
    return AB_OK;
}

/* ------------------------------------------------------------------ */
/* candidate list: insert_new_accelcand (src/accel_utils.c:387-469)    */
/* ------------------------------------------------------------------ */
/* The reference keeps an r-ordered singly linked list and walks it from
 * the head for every threshold crossing.  Here the list is an array: the
 * walk's stopping node ("first node with r >= rr, else the last node") is
 * found by binary search while the array is ordered, and by the same
 * linear walk otherwise (the reference can place a new candidate before
 * a last node exactly 15 bins lower, which breaks the ordering). */
struct ab_list {
    ab_cand *c;
    long long n, cap;
    int ordered;
};

ab_list *ab_list_new(void)
{
    ab_list *l = (ab_list *) calloc(1, sizeof(ab_list));
    if (l) l->ordered = 1;
    return l;
}

void ab_list_free(ab_list *l)
{
    if (!l) return;
    free(l->c);
    free(l);
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

static void list_check_order(ab_list *l, long long i)
{
    if (i > 0 && l->c[i - 1].r > l->c[i].r) l->ordered = 0;
    if (i + 1 < l->n && l->c[i].r > l->c[i + 1].r) l->ordered = 0;
}

int ab_list_insert(ab_list *l, float power, float sigma, int numharm,
                   double rr, double zz, double ww)
{
    if (list_reserve(l, l->n + 1)) return -1;
    ab_cand *c = l->c;
    if (l->n == 0) {
        set_cand(&c[0], power, sigma, numharm, rr, zz, ww);
        l->n = 1;
        return 1;
    }
    long long t;                       /* the walk's stopping node */
    if (l->ordered) {
        long long lo = 0, hi = l->n - 1;          /* search [0, n-1) */
        while (lo < hi) {
            long long mid = (lo + hi) / 2;
            if (c[mid].r < rr) lo = mid + 1; else hi = mid;
        }
        t = lo;
    } else {
        t = 0;
        while (t < l->n - 1 && c[t].r < rr) t++;
    }
    long long p = t - 1;
    int added = 0;
    double next_diff = fabs(rr - c[t].r);
    double prev_diff = p >= 0 ? fabs(rr - c[p].r) : AB_CLOSEST_R + 1.0;
    if (prev_diff < AB_CLOSEST_R) {
        if (c[p].sigma < sigma) {
            set_cand(&c[p], power, sigma, numharm, rr, zz, ww);
            list_check_order(l, p);
            added = 1;
        }
        if (next_diff < AB_CLOSEST_R && c[t].sigma < sigma) {
            if (added) {              /* the new candidate already replaced prev */
                memmove(&c[t], &c[t + 1], sizeof(ab_cand) * (size_t) (l->n - t - 1));
                l->n--;
            } else {
                set_cand(&c[t], power, sigma, numharm, rr, zz, ww);
                list_check_order(l, t);
                added = 1;
            }
        }
    } else if (next_diff < AB_CLOSEST_R) {
        if (c[t].sigma < sigma) {
            set_cand(&c[t], power, sigma, numharm, rr, zz, ww);
            list_check_order(l, t);
            added = 1;
        }
    } else {
        added = 1;
        long long at = (t == l->n - 1 && c[t].r < rr - AB_CLOSEST_R) ? l->n : t;
        memmove(&c[at + 1], &c[at], sizeof(ab_cand) * (size_t) (l->n - at));
        set_cand(&c[at], power, sigma, numharm, rr, zz, ww);
        l->n++;
        list_check_order(l, at);
    }
    return added;
}

long long ab_list_get(const ab_list *l, ab_cand *out, long long maxout)
{
    if (out)
        for (long long i = 0; i < l->n && i < maxout; i++) out[i] = l->c[i];
    return l->n;
}

/* LSD radix sort of (key, index) by the 62-bit key, 16 bits per pass. */
static int radix_order(const unsigned long long *keys, long long n, unsigned *order)
{
    unsigned *tmp = (unsigned *) malloc(sizeof(unsigned) * (size_t) n);
    unsigned long long *k0 = (unsigned long long *) malloc(sizeof(unsigned long long) * (size_t) n);
    unsigned long long *k1 = (unsigned long long *) malloc(sizeof(unsigned long long) * (size_t) n);
    size_t *cnt = (size_t *) malloc(sizeof(size_t) * 65536);
    if (!tmp || !k0 || !k1 || !cnt) {
        free(tmp); free(k0); free(k1); free(cnt);
        return AB_ERR_NOMEM;
    }
    for (long long i = 0; i < n; i++) { order[i] = (unsigned) i; k0[i] = keys[i]; }
    for (int pass = 0; pass < 4; pass++) {
        int sh = 16 * pass;
        memset(cnt, 0, sizeof(size_t) * 65536);
        for (long long i = 0; i < n; i++) cnt[(k0[i] >> sh) & 0xFFFF]++;
        size_t sum = 0;
        for (int d = 0; d < 65536; d++) { size_t c = cnt[d]; cnt[d] = sum; sum += c; }
        for (long long i = 0; i < n; i++) {
            size_t pos = cnt[(k0[i] >> sh) & 0xFFFF]++;
            k1[pos] = k0[i];
            tmp[pos] = order[i];
        }
        unsigned long long *kt = k0; k0 = k1; k1 = kt;
        memcpy(order, tmp, sizeof(unsigned) * (size_t) n);
    }
    free(tmp); free(k0); free(k1); free(cnt);
    return AB_OK;
}

/* Device hits carry (key, power, sigma); the key orders them as the
 * reference visits them (block, stage, w, z, r).  Replays search_ffdotpows'
 * per-hit work (src/accel_utils.c:1430-1442).  sigs may be NULL, in which
 * case candidate_sigma is evaluated here. */
int ab_replay_hits(const ab_obs *obs, unsigned long long *keys, float *pows, const float *sigs,
                   long long nhits, const double *startr_tab, long long ntab, ab_list *l)
{
    if (nhits <= 0) return AB_OK;
    unsigned *order = (unsigned *) malloc(sizeof(unsigned) * (size_t) nhits);
    if (!order) return AB_ERR_NOMEM;
    int rc = radix_order(keys, nhits, order);
    if (rc) { free(order); return rc; }
    long long cur_block = -1;
    ab_hgeom g = {0, 0, 0, 0};
    for (long long i = 0; i < nhits; i++) {
        unsigned long long k = keys[order[i]];
        int ri = (int) (k & 0xFFFF); k >>= AB_KEY_RBITS;
        int zi = (int) (k & 0xFFF); k >>= AB_KEY_ZBITS;
        int wi = (int) (k & 0x7F); k >>= AB_KEY_WBITS;
        int stage = (int) (k & 0x7); k >>= AB_KEY_SBITS;
        long long block = (long long) k;
        if (block >= ntab) { free(order); return AB_ERR_ARG; }
        if (block != cur_block) {
            /* the fundamental plane of the block (src/accel_utils.c:1034-1039) */
            double startr = startr_tab[block];
            g = ab_harm_geom(startr, startr + obs->rstep - AB_DR, 1, 1, obs->zlo, obs->wlo,
                             obs->corr_uselen);
            cur_block = block;
        }
        int numharm = 1 << stage;
        float pw = pows[order[i]];
        float sig = sigs ? sigs[order[i]]
                         : (float) ab_candidate_sigma(pw, numharm, (double) obs->numindep[stage]);
        double rr = (g.rlo + ri * (double) AB_DR) / (double) numharm;
        double zz = (g.zlo + zi * (double) AB_DZ) / (double) numharm;
        double ww = (g.wlo + wi * (double) AB_DW) / (double) numharm;
        if (ab_list_insert(l, pw, sig, numharm, rr, zz, ww) < 0) { free(order); return AB_ERR_NOMEM; }
    }
    free(order);
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
        int *o = info + 8 * k;
        o[0] = b->numharm; o[1] = b->harmnum; o[2] = b->nz; o[3] = b->nw;
        o[4] = b->fftlen_ref; o[5] = b->L; o[6] = b->hw0; o[7] = b->numrs_max;
    }
    return AB_OK;
}

long long ab_num_blocks_main(const ab_obs *obs) { return obs ? ab_num_blocks(obs) : -1; }
