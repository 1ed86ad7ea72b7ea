/*
 * accel_dropin.c -- libaccel_dropin.so: the reference's accel.h hot-path
 * functions (include/accel_dropin.h) over the B200 engine's C ABI.
 *
 * Each function keeps the reference's contract (arguments, return objects,
 * host layouts, list order, the .txtcand lines) and hands the arithmetic to
 * libaccel_b200.so: plane generation, harmonic sums and thresholding run on
 * the GPU; the planes come back into the caller's host arrays on every call,
 * so the reference's own code may read them at any point.  Objects the
 * engine needs to keep between calls (the block start an ffdotpows was made
 * for, the spectrum on the device, the device full plane) are held here.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "accel_b200.h"
#include "accel_dropin.h"
#include "ab_index.h"

/* glib (the list the reference's driver passes in) and libpresto's
 * accelcand destructor, resolved from the process (src/accel_utils.c:350-361) */
GSList *g_slist_alloc(void);
GSList *g_slist_remove_link(GSList *list, GSList *link_);
void g_slist_free_1(GSList *list);
void free_accelcand(void *data, void *user_data);

/* An ffdotpows made here, with the block start the engine needs to recompute
 * the subharmonic index maps of add_ffdotpows on the device. */
typedef struct {
    ffdotpows pub;              /* first: the caller sees a plain ffdotpows */
    double fullrlo;
} dropin_ffdot;

static ab_ctx *g_ctx;
static int g_spectrum_on_device;
static const fcomplex *g_spectrum_src;
static long long g_spectrum_bins;

static void die(const char *what, int rc)
{
    static const char *names[] = {"AB_OK", "AB_ERR_ARG", "AB_ERR_CUDA", "AB_ERR_NOMEM",
                                  "AB_ERR_OVERFLOW", "AB_ERR_STATE", "AB_ERR_BUDGET"};
    const char *name = (rc <= 0 && rc >= -6) ? names[-rc] : "?";
    fprintf(stderr, "\nlibaccel_dropin: %s failed: %s: %s\n", what, name,
            g_ctx ? ab_ctx_last_error(g_ctx) : "no engine context");
    exit(1);
}

static void *xmalloc(size_t n)
{
    void *p = malloc(n ? n : 1);
    if (!p) {
        perror("libaccel_dropin: malloc");
        exit(1);
    }
    return p;
}

static ab_ctx *ctx(void)
{
    if (!g_ctx) {
        const char *d = getenv("ACCEL_B200_DEVICE");
        int rc = ab_ctx_create(d ? atoi(d) : 0, &g_ctx);
        if (rc) die("ab_ctx_create", rc);
    }
    return g_ctx;
}

/* accelobs -> the engine's geometry record (the fields the hot path reads) */
static void engine_obs(const accelobs *o, ab_obs *a)
{
    memset(a, 0, sizeof(*a));
    a->N = o->N;
    a->numbins = o->numbins;
    a->lobin = o->lobin;
    a->highestbin = o->highestbin;
    a->maxkernlen = o->maxkernlen;
    a->corr_uselen = o->corr_uselen;
    a->fftlen = o->fftlen;
    a->numharmstages = o->numharmstages;
    a->numz = o->numz;
    a->numw = o->numw;
    a->numbetween = o->numbetween;
    a->inmem = o->inmem;
    a->norm_type = o->norm_type;
    a->rstep = (int) (o->corr_uselen * AB_DR);          /* src/accelsearch.c:85 */
    a->dt = o->dt;
    a->T = o->T;
    a->rlo = o->rlo;
    a->rhi = o->rhi;
    a->dr = o->dr;
    a->zlo = o->zlo;
    a->zhi = o->zhi;
    a->dz = o->dz;
    a->wlo = o->wlo;
    a->whi = o->whi;
    a->dw = o->dw;
    a->nph = o->nph;
    a->sigma = o->sigma;
    for (int s = 0; s < o->numharmstages && s < 6; s++) {
        a->powcut[s] = o->powcut[s];
        a->numindep[s] = o->numindep[s];
    }
    a->noharmpolish = !o->use_harmonic_polishing;
}

/* The spectrum goes to the device once per create_subharminfos: from the
 * mapped / in-memory transform, else read whole from the .fft file (file bin
 * 0 is bin obs->lobin, as read_fcomplex_file indexes it). */
static void ensure_spectrum(const accelobs *obs, const ab_obs *a)
{
    if (g_spectrum_on_device && g_spectrum_src == obs->fft && g_spectrum_bins == obs->numbins)
        return;
    const fcomplex *src = obs->fft;
    fcomplex *buf = NULL;
    if (!src) {
        if (!obs->fftfile) die("subharm_fderivs_vol (no spectrum: obs->fft and obs->fftfile "
                               "are both NULL)", AB_ERR_STATE);
        buf = (fcomplex *) xmalloc(sizeof(fcomplex) * (size_t) obs->numbins);
        if (fseeko(obs->fftfile, 0, SEEK_SET) != 0 ||
            fread(buf, sizeof(fcomplex), (size_t) obs->numbins, obs->fftfile) !=
                (size_t) obs->numbins)
            die("reading the .fft file", AB_ERR_ARG);
        src = buf;
    }
    int rc = ab_set_spectrum(ctx(), a, (const ab_fcomplex *) src);
    free(buf);
    if (rc) die("ab_set_spectrum", rc);
    g_spectrum_on_device = 1;
    g_spectrum_src = obs->fft;
    g_spectrum_bins = obs->numbins;
}

/* gen_f3Darr's layout: powers[w][z] row pointers into one contiguous block */
static float ***alloc_powers(int nw, int nz, int nr)
{
    float ***p = (float ***) xmalloc(sizeof(float **) * (size_t) nw);
    p[0] = (float **) xmalloc(sizeof(float *) * (size_t) nw * nz);
    p[0][0] = (float *) xmalloc(sizeof(float) * (size_t) nw * nz * nr);
    for (int w = 0; w < nw; w++) {
        p[w] = p[0] + (size_t) w * nz;
        for (int z = 0; z < nz; z++) p[w][z] = p[0][0] + ((size_t) w * nz + z) * nr;
    }
    return p;
}

static dropin_ffdot *new_ffdot(long long rlo, int zlo, int wlo, int nr, int nz, int nw)
{
    dropin_ffdot *d = (dropin_ffdot *) xmalloc(sizeof(*d));
    memset(d, 0, sizeof(*d));
    d->pub.rlo = rlo;
    d->pub.zlo = zlo;
    d->pub.wlo = wlo;
    d->pub.numrs = nr;
    d->pub.numzs = nz;
    d->pub.numws = nw;
    d->pub.powers = alloc_powers(nw, nz, nr);
    return d;
}

static ab_ffdotpows engine_plane(const ffdotpows *f)
{
    ab_ffdotpows e;
    e.rlo = f->rlo;
    e.zlo = f->zlo;
    e.wlo = f->wlo;
    e.numrs = f->numrs;
    e.numzs = f->numzs;
    e.numws = f->numws;
    e.powers = f->powers[0][0];
    e.capacity = (size_t) f->numws * f->numzs * f->numrs;
    return e;
}

subharminfo **create_subharminfos(accelobs *obs)
{
    ab_obs a;
    engine_obs(obs, &a);
    int rc = ab_prepare(ctx(), &a);                    /* device template banks */
    if (rc) die("create_subharminfos (device template banks)", rc);
    int nb = 0, info[9 * 64];
    rc = ab_bank_geometry(&a, &nb, info, 64);
    if (rc) die("ab_bank_geometry", rc);
    g_spectrum_on_device = 0;
    subharminfo **shis = (subharminfo **) xmalloc(sizeof(subharminfo *) * obs->numharmstages);
    /* shis[0][0] is the fundamental, shis[stage][harm - 1] harmonic harm/2^stage */
    shis[0] = (subharminfo *) xmalloc(2 * sizeof(subharminfo));
    for (int s = 1; s < obs->numharmstages && !obs->inmem; s++)
        shis[s] = (subharminfo *) xmalloc(sizeof(subharminfo) * (size_t) (1 << s));
    double dev_bytes = 0.0;
    for (int k = 0; k < nb; k++) {
        const int *g = info + 9 * k;
        const int numharm = g[0], harmnum = g[1], nz = g[2], nw = g[3], fftlen = g[4];
        int stage = 0;
        while ((1 << stage) < numharm) stage++;
        subharminfo *shi = &shis[stage][stage ? harmnum - 1 : 0];
        memset(shi, 0, sizeof(*shi));
        shi->numharm = numharm;
        shi->harmnum = harmnum;
        shi->numkern_zdim = nz;
        shi->numkern_wdim = nw;
        shi->numkern = nz * nw;
        shi->zmax = (nz - 1) / 2 * AB_DZ;
        shi->wmax = (nw - 1) / 2 * AB_DW;
        if (numharm > 1) {
            shi->rinds = (unsigned short *) xmalloc(sizeof(unsigned short) * obs->corr_uselen);
            shi->zinds = (unsigned short *) xmalloc(sizeof(unsigned short) * obs->corr_uselen);
        }
        shi->kern = (kernel **) xmalloc(sizeof(kernel *) * (size_t) nw);
        shi->kern[0] = (kernel *) xmalloc(sizeof(kernel) * (size_t) nw * nz);
        for (int wi = 0; wi < nw; wi++) {
            shi->kern[wi] = shi->kern[0] + (size_t) wi * nz;
            for (int zi = 0; zi < nz; zi++) {
                kernel *kn = &shi->kern[wi][zi];
                kn->z = -shi->zmax + zi * AB_DZ;
                kn->w = -shi->wmax + wi * AB_DW;
                kn->fftlen = fftlen;
                kn->numbetween = AB_NUMBETWEEN;
                kn->kern_half_width = ab_w_resp_halfwidth((double) kn->z, (double) kn->w);
                kn->numgoodbins = fftlen - 2 * AB_NUMBETWEEN * kn->kern_half_width;
                kn->data = NULL;           /* resident on the device */
            }
        }
        dev_bytes += (double) nz * nw * g[5] * sizeof(fcomplex);
        printf("  Harm %2d/%-2d: %6d templates on the GPU, %4d < z < %-4d, %5d < w < %-5d "
               "(%d-pt FFTs)\n", harmnum, numharm, nz * nw, -shi->zmax, shi->zmax, -shi->wmax,
               shi->wmax, g[5]);
    }
    printf("Total device RAM used by correlation kernels:  %.3f GB\n", dev_bytes / (1 << 30));
    return shis;
}

static void free_shi(subharminfo *shi)
{
    if (shi->kern) {
        free(shi->kern[0]);
        free(shi->kern);
    }
    free(shi->rinds);
    free(shi->zinds);
}

void free_subharminfos(accelobs *obs, subharminfo **shis)
{
    if (!shis) return;
    for (int s = 1; s < obs->numharmstages && !obs->inmem; s++) {
        for (int h = 1; h < (1 << s); h += 2) free_shi(&shis[s][h - 1]);
        free(shis[s]);
    }
    free_shi(&shis[0][0]);
    free(shis[0]);
    free(shis);
}

ffdotpows *subharm_fderivs_vol(int numharm, int harmnum, double fullrlo, double fullrhi,
                               subharminfo *shi, accelobs *obs)
{
    ab_obs a;
    engine_obs(obs, &a);
    ensure_spectrum(obs, &a);
    const ab_hgeom g = ab_harm_geom(fullrlo, fullrhi, numharm, harmnum, obs->zlo, obs->wlo,
                                    obs->corr_uselen);
    dropin_ffdot *d = new_ffdot(g.rlo, g.zlo, g.wlo, g.numrs, shi->numkern_zdim,
                                shi->numkern_wdim);
    d->fullrlo = fullrlo;
    ab_ffdotpows e = engine_plane(&d->pub);
    int rc = ab_subharm_fderivs_vol(ctx(), &a, numharm, harmnum, fullrlo, fullrhi, &e);
    if (rc) die("subharm_fderivs_vol", rc);
    /* the subharmonic index maps, as the reference leaves them in shi
       (src/accel_utils.c:1040-1053) */
    const double f = (double) harmnum / (double) numharm;
    if (numharm > 1 && !obs->inmem) {
        for (int ii = 0; ii < obs->corr_uselen; ii++)
            shi->rinds[ii] = (unsigned short) ab_rind(fullrlo, ii, f, g.rlo);
        for (int ii = 0; ii < obs->numz; ii++)
            shi->zinds[ii] = (unsigned short) ab_zind(obs->zlo, ii, f, g.zlo);
    }
    d->pub.rinds = shi->rinds;
    d->pub.zinds = shi->zinds;
    return &d->pub;
}

ffdotpows *copy_ffdotpows(ffdotpows *orig)
{
    const dropin_ffdot *o = (const dropin_ffdot *) orig;
    dropin_ffdot *d = new_ffdot(orig->rlo, orig->zlo, orig->wlo, orig->numrs, orig->numzs,
                                orig->numws);
    memcpy(d->pub.powers[0][0], orig->powers[0][0],
           sizeof(float) * (size_t) orig->numws * orig->numzs * orig->numrs);
    d->pub.rinds = orig->rinds;
    d->pub.zinds = orig->zinds;
    d->fullrlo = o->fullrlo;
    return &d->pub;
}

void free_ffdotpows(ffdotpows *ffd)
{
    if (!ffd) return;
    free(ffd->powers[0][0]);
    free(ffd->powers[0]);
    free(ffd->powers);
    free((dropin_ffdot *) ffd);
}

static void add_common(ffdotpows *fundamental, ffdotpows *subharmonic, int numharm, int harmnum,
                       int ptrs)
{
    ab_obs a;
    memset(&a, 0, sizeof(a));
    /* ab_add_ffdotpows reads only the search's z origin from the geometry */
    a.zlo = fundamental->zlo;
    ab_ffdotpows fe = engine_plane(fundamental), se = engine_plane(subharmonic);
    const double fullrlo = ((const dropin_ffdot *) subharmonic)->fullrlo;
    int rc = ptrs ? ab_add_ffdotpows_ptrs(ctx(), &a, &fe, &se, numharm, harmnum, fullrlo)
                  : ab_add_ffdotpows(ctx(), &a, &fe, &se, numharm, harmnum, fullrlo);
    if (rc) die(ptrs ? "add_ffdotpows_ptrs" : "add_ffdotpows", rc);
}

void add_ffdotpows(ffdotpows *fundamental, ffdotpows *subharmonic, int numharm, int harmnum)
{
    add_common(fundamental, subharmonic, numharm, harmnum, 0);
}

void add_ffdotpows_ptrs(ffdotpows *fundamental, ffdotpows *subharmonic, int numharm,
                        int harmnum)
{
    add_common(fundamental, subharmonic, numharm, harmnum, 1);
}

static void to_plane(ffdotpows *ffd, accelobs *obs, int trans)
{
    ab_obs a;
    engine_obs(obs, &a);
    ab_ffdotpows e = engine_plane(ffd);
    int rc = trans ? ab_fund_to_ffdotplane_trans(ctx(), &a, &e)
                   : ab_fund_to_ffdotplane(ctx(), &a, &e);
    if (rc) die(trans ? "fund_to_ffdotplane_trans" : "fund_to_ffdotplane", rc);
    if (!obs->ffdotplane) return;
    /* the caller's host plane, in the reference's layout */
    const long long rlen = (obs->highestbin + obs->corr_uselen) * (long long) AB_RDR;
    if (!trans) {
        for (int z = 0; z < ffd->numzs; z++)
            memcpy(obs->ffdotplane + (size_t) z * rlen + ffd->rlo * AB_RDR, ffd->powers[0][z],
                   sizeof(float) * (size_t) ffd->numrs);
    } else {
        float *out = obs->ffdotplane + (size_t) ffd->rlo * AB_RDR * ffd->numzs;
        for (int r = 0; r < ffd->numrs; r++)
            for (int z = 0; z < ffd->numzs; z++) *out++ = ffd->powers[0][z][r];
    }
}

void fund_to_ffdotplane(ffdotpows *ffd, accelobs *obs) { to_plane(ffd, obs, 0); }

void fund_to_ffdotplane_trans(ffdotpows *ffd, accelobs *obs) { to_plane(ffd, obs, 1); }

static void inmem_common(ffdotpows *fundamental, accelobs *obs, int numharm, int harmnum,
                         int trans)
{
    ab_obs a;
    engine_obs(obs, &a);
    ab_ffdotpows e = engine_plane(fundamental);
    int rc = trans ? ab_inmem_add_ffdotpows_trans(ctx(), &a, &e, numharm, harmnum)
                   : ab_inmem_add_ffdotpows(ctx(), &a, &e, numharm, harmnum);
    if (rc) die(trans ? "inmem_add_ffdotpows_trans" : "inmem_add_ffdotpows", rc);
}

void inmem_add_ffdotpows(ffdotpows *fundamental, accelobs *obs, int numharm, int harmnum)
{
    inmem_common(fundamental, obs, numharm, harmnum, 0);
}

void inmem_add_ffdotpows_trans(ffdotpows *fundamental, accelobs *obs, int numharm, int harmnum)
{
    inmem_common(fundamental, obs, numharm, harmnum, 1);
}

static accelcand *new_cand(float power, float sigma, int numharm, double r, double z, double w)
{
    accelcand *c = (accelcand *) xmalloc(sizeof(*c));
    memset(c, 0, sizeof(*c));
    c->power = power;
    c->sigma = sigma;
    c->numharm = numharm;
    c->r = r;
    c->z = z;
    c->w = w;
    return c;
}

#define CAND(node) ((accelcand *) (node)->data)

/* The reference's insertion rule (insert_new_accelcand,
 * src/accel_utils.c:387-469) on the caller's r-ordered GSList: a candidate
 * within ACCEL_CLOSEST_R bins of a neighbour replaces it when its sigma is
 * higher (and then drops a second close neighbour of lower sigma); one with
 * no close neighbour is linked in at its place. */
static GSList *insert_cand(GSList *list, float power, float sigma, int numharm, double rr,
                           double zz, double ww, int *added)
{
    *added = 0;
    if (!list) {
        GSList *node = g_slist_alloc();
        node->data = new_cand(power, sigma, numharm, rr, zz, ww);
        *added = 1;
        return node;
    }
    GSList *at = list, *before = NULL;
    while (at->next && CAND(at)->r < rr) {
        before = at;
        at = at->next;
    }
    const double d_at = fabs(rr - CAND(at)->r);
    const double d_before = before ? fabs(rr - CAND(before)->r) : AB_CLOSEST_R + 1.0;
    if (d_before < AB_CLOSEST_R) {
        if (CAND(before)->sigma < sigma) {
            free_accelcand(before->data, NULL);
            before->data = new_cand(power, sigma, numharm, rr, zz, ww);
            *added = 1;
        }
        if (d_at < AB_CLOSEST_R && CAND(at)->sigma < sigma) {
            free_accelcand(at->data, NULL);
            if (*added) {
                list = g_slist_remove_link(list, at);
                g_slist_free_1(at);
            } else {
                at->data = new_cand(power, sigma, numharm, rr, zz, ww);
                *added = 1;
            }
        }
        return list;
    }
    if (d_at < AB_CLOSEST_R) {
        if (CAND(at)->sigma < sigma) {
            free_accelcand(at->data, NULL);
            at->data = new_cand(power, sigma, numharm, rr, zz, ww);
            *added = 1;
        }
        return list;
    }
    GSList *node = g_slist_alloc();
    node->data = new_cand(power, sigma, numharm, rr, zz, ww);
    *added = 1;
    if (!at->next && CAND(at)->r < rr - AB_CLOSEST_R) {
        at->next = node;
        return list;
    }
    if (!before) {
        node->next = list;
        return node;
    }
    before->next = node;
    node->next = at;
    return list;
}

GSList *search_ffdotpows(ffdotpows *ffdot, int numharm, accelobs *obs, GSList *cands)
{
    static ab_cand *hits;
    static long long cap;
    ab_obs a;
    engine_obs(obs, &a);
    ab_ffdotpows e = engine_plane(ffdot);
    long long n = 0;
    int rc = ab_ffdot_hits(ctx(), &a, &e, numharm, hits, cap, &n);
    if (rc == AB_ERR_OVERFLOW) {
        free(hits);
        cap = n + n / 4 + 1024;
        hits = (ab_cand *) xmalloc(sizeof(ab_cand) * (size_t) cap);
        rc = ab_ffdot_hits(ctx(), &a, &e, numharm, hits, cap, &n);
    }
    if (rc) die("search_ffdotpows", rc);
    for (long long i = 0; i < n; i++) {
        const ab_cand *h = &hits[i];
        int added = 0;
        cands = insert_cand(cands, h->power, h->sigma, numharm, h->r, h->z, h->w, &added);
        if (added && !obs->dat_input)                  /* src/accel_utils.c:1443-1447 */
            fprintf(obs->workfile, "%-7.2f  %-7.4f  %-2d  %-14.4f  %-14.9f  %-10.4f %-10.4f\n",
                    h->power, h->sigma, numharm, h->r, h->r / obs->T, h->z, h->w);
    }
    return cands;
}
