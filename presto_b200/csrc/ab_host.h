/*
 * ab_host.h -- host-side C pieces of the engine shared with the CUDA
 * orchestration: template-bank geometry, the candidate list and the
 * replay of device threshold crossings in the reference's visit order.
 */
#ifndef AB_HOST_H
#define AB_HOST_H

#include "../../include/accel_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define AB_MAX_STAGES 6          /* numharm <= 32 (src/accel_utils.c:1635-1642) */
#define AB_MAX_BANKS 32          /* 1 + sum over stages of odd harmonics */

/* One template bank = one subharminfo (include/accel.h:107-118). */
typedef struct {
    int numharm, harmnum, stage;
    double f;                     /* harmnum / numharm */
    int zmax, wmax;               /* calc_required_z/w of the search maxima */
    int nz, nw, ntmpl;            /* numkern_zdim, numkern_wdim, numkern */
    int fftlen_ref;               /* the reference's FFT length (calc_fftlen) */
    int L, log2L;                 /* device FFT length (power of two) */
    int hw0;                      /* kern[0][0].kern_half_width (binoffset) */
    int numrs_max;                /* largest numrs over all blocks (row stride) */
    long long tmpl_off;           /* complex offset of the bank's templates */
    long long plane_off;          /* float offset inside one block's plane scratch */
    long long xhat_off;           /* complex offset inside one block's spectrum scratch */
    long long dtime_off;          /* complex offset of the block's normalised data
                                     (tensor-core correlation) */
    int sbm;                      /* blocks per device transform in the standard
                                     search (superblock height, >= 1) */
    int index;                    /* position in the bank set */
} ab_bank;

#define AB_MAX_SBM 8              /* superblock height limit */
#define AB_COST_SLOTS 16          /* transform cost table entries (by log2 L) */

typedef struct {
    int nbanks;
    ab_bank b[AB_MAX_BANKS];
    long long tmpl_total;         /* complex elements over all banks */
    long long plane_per_block;    /* floats of plane scratch per block */
    long long xhat_per_block;     /* complex elements of spectrum scratch per block */
    long long dtime_per_block;    /* complex elements of normalised data per block */
} ab_bankset;

/* Template-bank geometry for obs, in the reference's harmonic order:
 * (1,1), (2,1), (4,1), (4,3), (8,1), ... (src/accel_utils.c:240-288). */
int ab_bankset_init(const ab_obs *obs, ab_bankset *bs);
/* The same with measured per-template transform costs by log2 L
 * (AB_COST_SLOTS entries, <= 0 for unknown), which choose each bank's
 * transform length and superblock height. */
int ab_bankset_init_tuned(const ab_obs *obs, const double *cost_by_log2L, ab_bankset *bs);

/* Number of blocks of the main loop (src/accelsearch.c:187-224) and of the
 * in-memory low-frequency pre-pass (src/accelsearch.c:166-183). */
long long ab_num_blocks(const ab_obs *obs);
long long ab_num_preblocks(const ab_obs *obs);

int  ab_w_resp_halfwidth(double z, double w);
int  ab_dered_plan(long long numbins, int startwidth, int endwidth, double endfreq, double T,
                   int *blocks, long long maxblocks, long long *nblocks);
int  ab_next_good_fftlen(int n);
int  ab_fftlen_from_kernwidth(int kw);

/* Hit key packing: block:24 | stage:3 | w:7 | z:12 | r:16. */
#define AB_KEY_RBITS 16
#define AB_KEY_ZBITS 12
#define AB_KEY_WBITS 7
#define AB_KEY_SBITS 3
#define AB_KEY_BBITS 24

/* Replay sorted hits into the candidate list (insert_new_accelcand,
 * src/accel_utils.c:387-469, called from search_ffdotpows :1412-1452). */
typedef struct ab_list ab_list;
ab_list  *ab_list_new(void);
void      ab_list_free(ab_list *l);
int       ab_list_insert(ab_list *l, float power, float sigma, int numharm,
                         double rr, double zz, double ww);
long long ab_list_get(const ab_list *l, ab_cand *out, long long maxout);
/* work-file log: on != 0 records the reference's .txtcand line (T = the
 * observation's length, s) for every candidate an insertion adds */
void      ab_list_worklog(ab_list *l, int on, double T);
const char *ab_list_worklog_text(const ab_list *l, size_t *len);
/* Batches of at least this many crossings are replayed by clusters of r on
 * several threads (ab_list_replay_parallel), with the serial result. */
#define AB_REPLAY_PARALLEL_MIN 32768
int       ab_list_replay_parallel(ab_list *l, long long n, const float *pw, const float *sg,
                                  const int *nh, const double *rr, const double *zz,
                                  const double *ww, int nthreads);
int       ab_replay_hits(const ab_obs *obs, unsigned long long *keys, float *pows,
                         float *sigs, long long nhits, const double *startr_tab,
                         long long ntab, ab_list *l);
/* Start frequencies of the main-loop blocks, accumulated exactly as the
 * reference's driver does (startr += rstep). */
/* Birdie zapping (ab_zap.c): the span of bins [*span_lo, *span_hi) that the
 * -zaplist loop reads and writes (AB_ERR_ARG when a birdie's bins lie outside
 * the spectrum), and the loop over a host copy of that span (span[k] = bin
 * base + k). */
int       ab_zap_bounds(long long numbins, long long N, const double *lobins,
                        const double *hibins, int numbirds, long long *span_lo,
                        long long *span_hi);
int       ab_zapbirds_span(ab_fcomplex *span, long long base, long long numbins, long long N,
                           const double *lobins, const double *hibins, int numbirds,
                           int *numzapped);
void      ab_block_starts(const ab_obs *obs, double *out, long long n);
void      ab_preblock_starts(const ab_obs *obs, double *out, long long n);

#ifdef __cplusplus
}
#endif
#endif
