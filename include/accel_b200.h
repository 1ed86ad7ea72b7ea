/*
 * accel_b200.h -- C ABI of the B200 Fourier-domain acceleration/jerk search
 * engine (libaccel_b200.so).
 *
 * The engine is a drop-in for the hot path of PRESTO's accelsearch:
 * template generation (create_subharminfos), plane generation
 * (subharm_fderivs_vol), harmonic summing (add_ffdotpows,
 * inmem_add_ffdotpows) and threshold search (search_ffdotpows).  Plain
 * pointers and sizes only; no CUDA or torch types cross this boundary.
 * Every call returns AB_OK (0) or a negative AB_ERR_* code; the message of
 * the last error on a context is available from ab_ctx_last_error().
 *
 * Reference interface each entry point replaces (PRESTO 6.0.1):
 *   ab_obs_init             create_accelobs           src/accel_utils.c:1455-1805
 *                                                     (geometry/thresholds part)
 *   ab_prepare              create_subharminfos       src/accel_utils.c:240-288
 *   ab_subharm_fderivs_vol  subharm_fderivs_vol       src/accel_utils.c:1024-1198
 *   ab_add_ffdotpows        add_ffdotpows             src/accel_utils.c:1261-1282
 *   ab_fund_to_ffdotplane   fund_to_ffdotplane        src/accel_utils.c:1219-1233
 *   ab_inmem_add_ffdotpows  inmem_add_ffdotpows       src/accel_utils.c:1312-1361
 *   ab_search_ffdotpows     search_ffdotpows          src/accel_utils.c:1412-1452
 *   ab_search               the block/stage loop of   src/accelsearch.c:161-224
 *   ab_sort_cands           sort_accelcands           src/accel_utils.c:364-384
 *   ab_eliminate_harmonics  eliminate_harmonics       src/accel_utils.c:472-549
 *   ab_candidate_sigma      candidate_sigma           src/characteristics.c:526-546
 *   ab_power_for_sigma      power_for_sigma           src/characteristics.c:549-559
 *   ab_gen_response         gen_w_response/gen_z_response/gen_r_response
 *                                                     src/responses.c:159-418
 *   ab_write_accelfile      output_fundamentals +     src/accel_utils.c:666-966
 *                           output_harmonics
 */
#ifndef ACCEL_B200_H
#define ACCEL_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AB_OK              0
#define AB_ERR_ARG        -1   /* invalid argument or unsupported geometry */
#define AB_ERR_CUDA       -2   /* CUDA runtime error */
#define AB_ERR_NOMEM      -3   /* device or host allocation failed */
#define AB_ERR_OVERFLOW   -4   /* hit buffer or output array too small */
#define AB_ERR_STATE      -5   /* call out of order (e.g. no spectrum) */
#define AB_ERR_BUDGET     -6   /* request exceeds the HBM budget */

/* fcomplex: include/ransomfft.h:13-16 (interleaved re, im) */
typedef struct { float r, i; } ab_fcomplex;

/* Search options that reach the hot path; the fields and defaults mirror
 * the accelsearch command line (clig/accelsearch_cmd.cli,
 * src/accelsearch_cmd.c:22-61).  Use ab_params_default() to fill them. */
typedef struct {
    long long N;          /* time-series samples (.inf N) */
    double dt;            /* sample time, s (.inf dt) */
    long long numbins;    /* complex bins in the .fft */
    int zmax, wmax, wmaxP;/* -zmax, -wmax (wmaxP: -wmax given) */
    int numharm;          /* -numharm (power of two, <= 32) */
    float sigma;          /* -sigma */
    double flo, fhi; int floP, fhiP;
    double rlo, rhi; int rloP, rhiP;
    long long lobin;      /* -lobin */
    int inmemP;           /* -inmem */
    float nph;            /* > 0: -photon normalisation with this level */
    int locpowP;          /* -locpow: double-tophat local-power normalisation */
    int noharmpolishP;    /* -noharmpolish: polish each harmonic on its own */
} ab_params;

/* accelobs geometry (include/accel.h:37-81), hot-path fields only. */
typedef struct {
    long long N, numbins, lobin, highestbin;
    int maxkernlen, corr_uselen, fftlen, numharmstages, numz, numw;
    int numbetween, inmem, norm_type, rstep;
    double dt, T, rlo, rhi, dr, zlo, zhi, dz, wlo, whi, dw;
    float nph, sigma;
    float powcut[6];
    long long numindep[6];
    int noharmpolish;             /* 1: -noharmpolish, each harmonic polished alone
                                     (use_harmonic_polishing = 0, src/accel_utils.c:1489-1494);
                                     0, the default, in a zero-filled ab_obs */
} ab_obs;

/* accelcand search fields (include/accel.h:83-95). */
typedef struct {
    float power, sigma;
    int numharm;
    double r, z, w;
} ab_cand;

/* ffdotpows (include/accel.h:120-130) with powers[numws][numzs][numrs]
 * in caller-owned host memory. */
typedef struct {
    long long rlo;
    int zlo, wlo, numrs, numzs, numws;
    float *powers;
    size_t capacity;      /* floats available at powers */
} ab_ffdotpows;

typedef struct ab_ctx ab_ctx;

void ab_params_default(ab_params *p);

/* Context: one per device and host thread. */
int  ab_ctx_create(int device, ab_ctx **out);
void ab_ctx_destroy(ab_ctx *ctx);
const char *ab_ctx_last_error(const ab_ctx *ctx);
void *ab_ctx_stream(ab_ctx *ctx);                 /* cudaStream_t of the context */
int  ab_ctx_set_hbm_budget(ab_ctx *ctx, size_t bytes);

/* Correlation path of the context's searches and drop-ins (replaces the
 * FFTW multiply / inverse transform of subharm_fderivs_vol,
 * src/accel_utils.c:1140-1193, by one of two device evaluations):
 *   AB_CORR_FFT            FP32 radix-16 FFTs fused with the template
 *                          multiply and power (default);
 *   AB_CORR_TC_SPLIT_BF16  the banded template product as a complex
 *                          contraction on the tensor cores, operands split
 *                          into BF16 hi + lo parts, FP32 accumulation;
 *   AB_CORR_TC_SPLIT_FP16  the same with FP16 hi + lo parts (11 significant
 *                          bits each instead of 8: ~2^-22 relative products;
 *                          normalised amplitudes must stay below 65504, i.e.
 *                          powers below ~4e9 times the block's noise level).
 * The reference has no counterpart (it has one path). */
#define AB_CORR_FFT            0
#define AB_CORR_TC_SPLIT_BF16  1
#define AB_CORR_TC_SPLIT_FP16  2
int  ab_ctx_set_corr_path(ab_ctx *ctx, int path);

/* Transform schedule (no counterpart in the reference, whose FFT length per
 * harmonic is calc_fftlen's, src/accel_utils.c:137-150).  The whole-spectrum
 * search correlates each bank with a device FFT of length L (512..8192) that
 * serves m consecutive blocks (1..8, only where the reference's own transform
 * does not wrap); L and m minimise the correlation cost per block under a
 * process-wide table of costs per template and transform, indexed by log2 L
 * (AB_COST_SLOTS = 16 entries; a length whose entry is <= 0 is not used for
 * superblocks).  The library starts with a table measured on B200 for 512 to
 * 4096 points; ab_autotune re-measures those on the context's device and
 * installs them (costs_out may be NULL).  Set the table before creating the
 * banks a search, ab_bank_geometry or ab_fderivs_vol_noalloc rely on: the
 * template length follows it. */
int  ab_set_transform_costs(const double *costs, int n);
int  ab_get_transform_costs(double *costs, int n);
int  ab_autotune(ab_ctx *ctx, double *costs_out, int n);

/* Geometry + thresholds (create_accelobs).  Host only. */
int ab_obs_init(const ab_params *p, ab_obs *obs);

/* Template-bank geometry of obs in the reference's harmonic order (host
 * only).  info[9*k ..] = numharm, harmnum, numkern_zdim, numkern_wdim,
 * reference fftlen, device FFT length, kernel half width, largest numrs,
 * blocks per device transform in the whole-spectrum search. */
int ab_bank_geometry(const ab_obs *obs, int *nbanks, int *info, int maxbanks);

/* Number of blocks of the main search loop (src/accelsearch.c:187-224). */
long long ab_num_blocks_main(const ab_obs *obs);

/* Template banks for obs (create_subharminfos); cached on the context. */
int ab_prepare(ab_ctx *ctx, const ab_obs *obs);

/* Whole-spectrum search: every block and harmonic stage of the main loop.
 * fft holds obs->numbins bins; fft_on_device != 0 means fft is a device
 * pointer, else a host pointer copied in by the call.  Candidates come back
 * in the order the reference's list holds them (increasing r).
 * first_block/max_blocks restrict the main loop (max_blocks < 0: all). */
int ab_search(ab_ctx *ctx, const ab_obs *obs, const ab_fcomplex *fft, int fft_on_device,
              long long first_block, long long max_blocks,
              ab_cand *cands, long long maxcands, long long *numcands);

/* Candidate list of the last ab_search (all of it, whatever maxcands was). */
int ab_last_cands(ab_ctx *ctx, ab_cand *out, long long maxout, long long *numcands);

/* Raw threshold crossings of the last ab_search, in reference visit order
 * (block, stage, w, z, r): block ordinal, stage, w index, z index, r index,
 * power.  Returns the count through *numhits. */
int ab_last_hits(ab_ctx *ctx, long long *block, int *stage, int *wi, int *zi, int *ri,
                 float *power, long long maxhits, long long *numhits);

/* Per-function drop-ins (one block at a time).  ab_set_spectrum uploads the
 * .fft bins used by later ab_subharm_fderivs_vol calls; the in-memory full
 * f-fdot plane (accelobs.ffdotplane) stays resident on the device and is
 * filled by ab_fund_to_ffdotplane.  fullrhi must equal
 * fullrlo + rstep - ACCEL_DR, as in the reference's driver loop. */
int ab_set_spectrum(ab_ctx *ctx, const ab_obs *obs, const ab_fcomplex *fft_host);
int ab_subharm_fderivs_vol(ab_ctx *ctx, const ab_obs *obs, int numharm, int harmnum,
                           double fullrlo, double fullrhi, ab_ffdotpows *out);
int ab_add_ffdotpows(ab_ctx *ctx, const ab_obs *obs, ab_ffdotpows *fund,
                     const ab_ffdotpows *sub, int numharm, int harmnum, double fullrlo);
int ab_fund_to_ffdotplane(ab_ctx *ctx, const ab_obs *obs, const ab_ffdotpows *fund);
int ab_inmem_add_ffdotpows(ab_ctx *ctx, const ab_obs *obs, ab_ffdotpows *fund,
                           int numharm, int harmnum);

/* The -otheropt forms the reference's driver selects instead
 * (src/accelsearch.c:145-159): add_ffdotpows_ptrs (src/accel_utils.c:1284-1309),
 * fund_to_ffdotplane_trans (:1236-1250) and inmem_add_ffdotpows_trans
 * (:1364-1409) compute the same sums as the plain forms over an [r][z] host
 * plane.  The engine's full plane is its own device array, so these take the
 * plain forms' arguments and give their results. */
int ab_add_ffdotpows_ptrs(ab_ctx *ctx, const ab_obs *obs, ab_ffdotpows *fund,
                          const ab_ffdotpows *sub, int numharm, int harmnum, double fullrlo);
int ab_fund_to_ffdotplane_trans(ab_ctx *ctx, const ab_obs *obs, const ab_ffdotpows *fund);
int ab_inmem_add_ffdotpows_trans(ab_ctx *ctx, const ab_obs *obs, ab_ffdotpows *fund,
                                 int numharm, int harmnum);

/* copy_ffdotpows (src/accel_utils.c:1200-1217): geometry and powers of src
 * into dst, whose powers array is the caller's (dst->capacity floats).
 * Host only. */
int ab_copy_ffdotpows(const ab_ffdotpows *src, ab_ffdotpows *dst);

/* get_fourier_amplitudes (src/accel_utils.c:993-1022): numbins bins from
 * lobin of the spectrum fft (obs->numbins bins starting at obs->lobin) into
 * out, zero where the window runs off either end.  Host only. */
int ab_get_fourier_amplitudes(const ab_obs *obs, const ab_fcomplex *fft, long long lobin,
                              int numbins, ab_fcomplex *out);

/* Candidate list (the GSList of accelcand built by search_ffdotpows). */
typedef struct ab_list ab_candlist;
ab_candlist *ab_candlist_new(void);
void ab_candlist_free(ab_candlist *l);
long long ab_candlist_get(const ab_candlist *l, ab_cand *out, long long maxout);
/* insert_new_accelcand (src/accel_utils.c:387-469); returns 1 if added. */
int ab_candlist_insert(ab_candlist *l, float power, float sigma, int numharm,
                       double r, double z, double w);
int ab_search_ffdotpows(ab_ctx *ctx, const ab_obs *obs, const ab_ffdotpows *ffd,
                        int numharm, ab_candlist *list);
/* The threshold crossings search_ffdotpows visits (src/accel_utils.c:1412-1452),
 * for callers that keep their own candidate list: every cell of ffd above
 * obs->powcut[stage of numharm], in the reference's visit order (w, z, r),
 * as (power, candidate_sigma, numharm, r, z, w) of the candidate it would
 * insert.  *numhits gets the count; AB_ERR_OVERFLOW when it exceeds maxout
 * (out may be NULL with maxout 0 to count). */
int ab_ffdot_hits(ab_ctx *ctx, const ab_obs *obs, const ab_ffdotpows *ffd, int numharm,
                  ab_cand *out, long long maxout, long long *numhits);

/* The .txtcand work file: search_ffdotpows writes one line per candidate an
 * insertion adds, "%-7.2f  %-7.4f  %-2d  %-14.4f  %-14.9f  %-10.4f %-10.4f"
 * of power, sigma, numharm, r, r / T, z, w (src/accel_utils.c:1443-1447),
 * in search order, for .fft input.
 *   ab_set_worklog      on != 0: later ab_search calls record those lines;
 *   ab_last_worklog     the last ab_search's lines: *len bytes; up to
 *                       cap - 1 of them copied to out, NUL-terminated;
 *   ab_candlist_set_worklog / ab_candlist_worklog  the same for a list that
 *                       ab_search_ffdotpows / ab_candlist_insert fill (T the
 *                       observation's length, s); the second returns the
 *                       length and copies as ab_last_worklog does. */
int ab_set_worklog(ab_ctx *ctx, int on);
int ab_last_worklog(ab_ctx *ctx, char *out, size_t cap, size_t *len);
int ab_candlist_set_worklog(ab_candlist *l, int on, double T);
long long ab_candlist_worklog(const ab_candlist *l, char *out, size_t cap);

/* Stage sums of one block of the last ab_search configuration, for parity
 * checks: out[stage][numws][numzs][numrs] after each stage. */
int ab_block_stage_sums(ab_ctx *ctx, const ab_obs *obs, const ab_fcomplex *fft_host,
                        long long block, float *out, size_t capacity);

/* Template generation (kernel set a) on the device, FP64, returned as FP32
 * (gen_w_response(roffset, numbetween, z, w, numkern)). */
int ab_gen_response(ab_ctx *ctx, double roffset, int numbetween, double z, double w,
                    int numkern, ab_fcomplex *out);

/* The FFT'd template (w index wi, z index zi) of bank (numharm, harmnum)
 * as stored on the device, and its device FFT length. */
int ab_bank_kernel(ab_ctx *ctx, const ab_obs *obs, int numharm, int harmnum, int wi, int zi,
                   ab_fcomplex *out, int maxlen, int *fftlen_dev);

/* Plane generation for one block and one harmonic that allocates no memory.
 * No counterpart in the reference: it is ab_subharm_fderivs_vol for callers
 * that cannot call cudaMalloc (pipelines that reserve all device memory at
 * start-up, hosts whose device memory belongs to another allocator, or
 * stream-ordered code where an allocation would synchronise the device).
 * Inputs and outputs are device pointers owned by the caller: d_fft holds
 * obs->numbins bins; d_templates the bank of harmonic harmnum/numharm as
 * [numkern_wdim][numkern_zdim][L] FFT'd templates (L and the dimensions from
 * ab_bank_geometry, each template as ab_bank_kernel returns it) in a buffer
 * of templates_capacity complex values (AB_ERR_ARG when the bank needs more,
 * e.g. after ab_set_transform_costs or ab_autotune changed L); d_powers
 * receives powers[numws][numzs][numrs] (capacity in floats, else
 * AB_ERR_OVERFLOW).  The block starts at fullrlo and ends at
 * fullrlo + rstep - 0.5.  Work is queued on `stream` (a cudaStream_t, NULL
 * for the default stream) of the calling thread's current device; the call
 * does not wait for it.  A CUDA error already pending on the calling thread
 * returns AB_ERR_STATE with nothing launched and the error left in place.
 * The engine's intermediates live in one static device array of 192 KiB
 * that every GPU loading the library keeps until exit, so the bank must need
 * at most 8192 correlation work items and a data spectrum of at most 4096
 * points, else AB_ERR_BUDGET (and a line on stderr); every bank that
 * ab_bank_geometry accepts fits (at most ~4600 items and 2048 points).  The
 * array is shared by all calls and keeps the last call's contents; every
 * word a call reads is written earlier in the same call, so nothing needs
 * clearing, but calls whose GPU work overlaps (different streams, threads)
 * race on it.  The first call in each CUDA context looks up the array's
 * address (cudaGetSymbolAddress) and caches it under the context's ID, so a
 * context created after a cudaDeviceReset gets a fresh lookup: make that
 * first call before any stream capture.
 * meta_out (optional) receives the plane's rlo, zlo, wlo and sizes. */
int ab_fderivs_vol_noalloc(const ab_obs *obs, int numharm, int harmnum, double fullrlo,
                           const ab_fcomplex *d_fft, const ab_fcomplex *d_templates,
                           size_t templates_capacity, float *d_powers, size_t powers_capacity,
                           void *stream, ab_ffdotpows *meta_out);

/* Batched and served searches (no counterpart in the reference, whose
 * accelsearch searches one spectrum per process: src/accelsearch.c:44-316).
 * A pool of nworkers engine contexts on one device, each on its own host
 * thread and stream.  Requests queue in arrival order; a free worker takes
 * the head request once its device-memory footprint (in-memory plane plus
 * spectrum, on top of every worker's fixed scratch) fits hbm_budget (0: 80 %
 * of the free memory), so requests arriving while others run are admitted as
 * workers and memory free up, and their kernels overlap on the GPU.  Each
 * result equals ab_search of that request alone.  ab_pool_submit copies the
 * spectrum (p->numbins bins); ab_pool_wait blocks for the result (out NULL:
 * count only, the result is kept), then frees it; latency = submit to done. */
typedef struct ab_pool ab_pool;
int  ab_pool_create(int device, int nworkers, size_t hbm_budget, ab_pool **out);
void ab_pool_destroy(ab_pool *pool);
const char *ab_pool_last_error(const ab_pool *pool);
/* The correlation path (AB_CORR_*) of every worker, set while no request is
 * queued (AB_ERR_STATE otherwise). */
int  ab_pool_set_corr_path(ab_pool *pool, int path);
int  ab_pool_submit(ab_pool *pool, const ab_params *p, const ab_fcomplex *fft, long long *ticket);
int  ab_pool_wait(ab_pool *pool, long long ticket, ab_cand *out, long long maxout,
                  long long *numcands, double *latency_ms);
/* completed requests, p50/p99 latency (ms) and first start to last finish. */
int  ab_pool_stats(ab_pool *pool, long long *completed, double *p50_ms, double *p99_ms,
                   double *busy_ms);
int  ab_pool_reset_stats(ab_pool *pool);

/* Tensor-core self-test (no counterpart in the reference): C[128][N] =
 * A[128][K] . B[N][K]^T through tcgen05 BF16 MMAs with FP32 accumulation in
 * tensor memory, operands split into hi + lo BF16 parts when split != 0 (the
 * arithmetic of the split-precision correlation).  Host arrays; K % 16 == 0,
 * K <= 256, N % 16 == 0, 16 <= N <= 256. */
int ab_tc_gemm(ab_ctx *ctx, const float *A, const float *B, float *C, int N, int K, int split);

/* Candidate polishing: optimize_accelcand (src/accel_utils.c:552-626) with
 * the reference's default harmonic polishing, every candidate at once on the
 * device: max_rz_arr_harmonics (src/maximize_rz.c:173-228) for an
 * acceleration search (obs->numw == 0), max_rzw_arr_harmonics
 * (src/maximize_rzw.c:81-191) for a jerk search (obs->numw > 0).  fft holds
 * obs->numbins bins (device pointer when fft_on_device != 0).  out[k]
 * receives the optimised r, z, w of each harmonic of cands[k], its raw power
 * and its rderivs (include/presto.h:160-168).  AB_ERR_ARG for a jerk
 * candidate whose responses need chirps above 2^17 samples. */
#define AB_POLISH_MAX_HARM 32
typedef struct {
    double pow, phs, dpow, dphs, d2pow, d2phs, locpow;
} ab_rderivs;
typedef struct {
    int numharm;
    double pows[AB_POLISH_MAX_HARM];
    double hirs[AB_POLISH_MAX_HARM], hizs[AB_POLISH_MAX_HARM], hiws[AB_POLISH_MAX_HARM];
    ab_rderivs derivs[AB_POLISH_MAX_HARM];
} ab_polished;
int ab_optimize_cands(ab_ctx *ctx, const ab_obs *obs, const ab_fcomplex *fft, int fft_on_device,
                      const ab_cand *cands, long long n, ab_polished *out);

/* Candidate properties (Middleditch, Deich & Kulkarni 1993) and the .cand
 * file.  ab_fourierprops has fourierprops' members and layout
 * (include/presto.h:170-188): the reference's .cand file is an array of it
 * written raw (src/accelsearch.c:282-284), so an array of n of these is that
 * file's content.  ab_rzwerrs is rzwerrs (include/presto.h:233-246).
 *   ab_calc_props    calc_props (src/characteristics.c:195-264); AB_ERR_ARG
 *                    where the reference exits (|pow| or locpow < 1e-14);
 *   ab_calc_rzwerrs  calc_rzwerrs (src/characteristics.c:353-392); AB_ERR_ARG
 *                    for T <= 0;
 *   ab_cand_props    per polished candidate, the fundamental's properties
 *                    at the search's (r, z, w) with the reference's error
 *                    overrides ACCEL_DR, ACCEL_DZ, ACCEL_DW / numharm
 *                    (src/accelsearch.c:261-272). */
typedef struct {
    double r;
    float rerr;
    double z;
    float zerr;
    double w;
    float werr;
    float pow, powerr, sig, rawpow, phs, phserr, cen, cenerr, pur, purerr, locpow;
} ab_fourierprops;
typedef struct {
    double p, pd, pdd, f, fd, fdd;
    float perr, pderr, pdderr, ferr, fderr, fdderr;
} ab_rzwerrs;
int ab_calc_props(const ab_rderivs *d, double r, double z, double w, ab_fourierprops *out);
int ab_calc_rzwerrs(const ab_fourierprops *props, double T, ab_rzwerrs *out);
int ab_cand_props(const ab_cand *cands, const ab_polished *pol, long long n, ab_fourierprops *out);

/* The text candidate file <root>_ACCEL_<zmax>[_JERK_<wmax>]: the
 * fundamentals table (output_fundamentals, src/accel_utils.c:666-841) and
 * the harmonics table (output_harmonics, src/accel_utils.c:844-966) of n
 * sorted, polished candidates (out of ab_optimize_cands), with the .inf at
 * inf_path appended as the reference's "cat <root>.inf >>" does (NULL or an
 * unreadable file: nothing appended).  Notes are the candidates' own
 * (compare_rzw_cands, src/accel_utils.c:105-134); the pulsar-catalogue notes
 * of an observation with a telescope name are not made.  AB_ERR_ARG where
 * the reference exits (a power or local power ~ 0, T <= 0, a value
 * nice_output_2 cannot format) or the file cannot be written; nothing is
 * written then.
 *   ab_nice_output_1 / ab_nice_output_2  nice_output_1 / nice_output_2
 *   (src/output.c:6-210) into out[outlen]: val(err) with a one- or two-digit
 *   error, left-justified for len == 0, else right-justified to len; the
 *   string length, or AB_ERR_ARG (no room, or nice_output_2's undefined
 *   case). */
int ab_write_accelfile(const char *path, const ab_obs *obs, const ab_cand *cands,
                       const ab_polished *pol, long long n, const char *inf_path);
int ab_nice_output_1(char *out, size_t outlen, double val, double err, int len);
int ab_nice_output_2(char *out, size_t outlen, double val, double err, int len);

/* The time-series input of create_accelobs (.dat files,
 * src/accel_utils.c:1516-1563) on the device:
 *   ab_realfft       realfft(data, n, -1) (src/fastffts.c:163-246): n float
 *                    samples to n/2 bins, bin 0 = (DC, Nyquist); n/2 must be
 *                    a power of two from 512 to 8192 or from 65536 to 2^26;
 *   ab_deredden      deredden (src/misc_utils.c:912-1067) in place;
 *   ab_series_to_fft both, with accelsearch's arguments (6, 200, 0.5/dt,
 *                    n dt).
 * *_on_device flags say whether each pointer is a device pointer. */
int ab_realfft(ab_ctx *ctx, const float *series, long long n, int series_on_device, ab_fcomplex *out,
               int out_on_device);
int ab_deredden(ab_ctx *ctx, ab_fcomplex *fft, long long numbins, int startwidth, int endwidth,
                double endfreq, double T, int fft_on_device);
int ab_series_to_fft(ab_ctx *ctx, const float *series, long long n, double dt, int series_on_device,
                     ab_fcomplex *out, int out_on_device);

/* Birdie zapping of -zaplist (src/accelsearch.c:87-110; accelsearch zaps
 * only a spectrum it holds in memory, i.e. one made from a .dat time
 * series):
 *   ab_read_zaplist   get_birdies (src/birdzap.c:6-88): "<freq> <width>"
 *                     lines in Hz (Doppler shifted by 1 + baryv), "B<freq>
 *                     <width>" barycentric, '#' comments; each birdie at
 *                     least one bin wide; sorted by low bin.  *numbirds gets
 *                     the count (AB_ERR_OVERFLOW above maxbirds).  Blank or
 *                     unparseable lines are skipped.
 *   ab_zapbirds       the reference's loop over the sorted list: birdies
 *                     from N/2 on are dropped, high edges clipped to N/2 - 1,
 *                     each zapped as zapbirds (src/zapping.c:58-150) does --
 *                     the bins replaced by exponential-power, uniform-phase
 *                     noise at the local mean power (the median of 200
 *                     bins each side, 100 bins out, over ln 2), drawn from
 *                     GSL's MT19937 seeded with 1 (a fresh stream per call,
 *                     as per accelsearch run).  fft_on_device: fft is a
 *                     device pointer; only the bins read and written cross
 *                     the bus.  *numzapped (optional) counts the birdies
 *                     zapped (those with no room for either window are
 *                     skipped, as the reference does with a warning).
 *   ab_zapbirds_host  the same on a host spectrum, no context needed.
 *   ab_mt19937_output the k-th (from 1) 32-bit output of that generator
 *                     for a seed (GSL seeding; seed 0 means 4357), to check
 *                     it against the generator's published outputs. */
int ab_read_zaplist(const char *path, double T, double baryv, double *lobins, double *hibins,
                    int maxbirds, int *numbirds);
int ab_zapbirds(ab_ctx *ctx, ab_fcomplex *fft, int fft_on_device, long long numbins, long long N,
                const double *lobins, const double *hibins, int numbirds, int *numzapped);
int ab_zapbirds_host(ab_fcomplex *fft, long long numbins, long long N, const double *lobins,
                     const double *hibins, int numbirds, int *numzapped);
unsigned int ab_mt19937_output(unsigned long seed, long long k);

/* Subband dedispersion, the producer of accelsearch's DM trials (prepsubband,
 * src/prepsubband.c:365-450, src/dispersion.c:54-232; no reference
 * counterpart for the whole-array form: prepsubband streams blocks of the
 * raw data through the same sums).  data: nspec spectra of nchan channels,
 * time-major (all channels of a sample together, channel 0 the lowest
 * frequency lofreq MHz, chanwidth > 0 MHz apart), as floats; dt the sample
 * time (s).  Channels are summed into nsub subbands with the delays of the
 * DMs' mean (subband_search_delays, rounded to samples), the subbands are
 * downsampled by downsamp (averages, prepsubband -downsamp), then each DM
 * d sums the subbands shifted by its offsets (subband_delays relative to the
 * top subband, rounded to downsampled samples): out[d][u] for
 * u < nspec / downsamp, DM-major.  Samples past the end read zero (the
 * reference's zero-padded last block).  Every output element is summed in
 * the reference's order, so it is the reference's float result.
 *   ab_dedisp_delays  the channel delays (nchan ints) and subband offsets
 *                     (ndm x nsub ints) it uses, host only;
 *   ab_dedisperse     the dedispersion; *_on_device flags say whether data
 *                     and out are device pointers. */
int ab_dedisp_delays(int nchan, double lofreq, double chanwidth, double dt, int nsub,
                     const double *dms, int ndm, int downsamp, int *chan_delay, int *sub_offset);
int ab_dedisperse(ab_ctx *ctx, const float *data, int data_on_device, long long nspec, int nchan,
                  double lofreq, double chanwidth, double dt, int nsub, const double *dms, int ndm,
                  int downsamp, float *out, int out_on_device);

/* The DM-trial pipeline on the device (prepsubband, then accelsearch on each
 * trial's .dat, src/accel_utils.c:1552-1562 for the series): the spectra are
 * dedispersed as ab_dedisperse does, each trial becomes a spectrum as
 * ab_series_to_fft makes it (realfft + deredden), and that spectrum is
 * searched as ab_search searches it, without the trials or their spectra
 * leaving the device.  obs must describe the trials: N = (nspec / downsamp)
 * rounded down to even (an odd last sample is dropped, as realfft needs an
 * even length) and dt = dt * downsamp.  Trial d's candidates, in ab_search's
 * order, are cands[first[d] .. first[d + 1]) (first: ndm + 1 offsets, always
 * filled); AB_ERR_OVERFLOW when they exceed maxcands (cands may be NULL to
 * count them).  ab_last_cands afterwards holds the last trial's. */
int ab_search_dedispersed(ab_ctx *ctx, const float *data, int data_on_device, long long nspec,
                          int nchan, double lofreq, double chanwidth, double dt, int nsub,
                          const double *dms, int ndm, int downsamp, const ab_obs *obs,
                          ab_cand *cands, long long maxcands, long long *first);

/* Host-side statistics and candidate-list helpers. */
double ab_candidate_sigma(double power, int numsum, double numtrials);
double ab_power_for_sigma(double sigma, int numsum, double numtrials);
double ab_chi2_logp(double chi2, double dof);
double ab_equivalent_gaussian_sigma(double logp);
int  ab_sort_cands(ab_cand *cands, long long n);
long long ab_eliminate_harmonics(ab_cand *cands, long long n);
/* Half-width in bins of the (z, w) response, w_resp_halfwidth with LOWACC
 * (src/responses.c:49-84; z_resp_halfwidth :27-47 when w = 0). */
int  ab_w_resp_halfwidth(double z, double w);

/* Kernel timing (CUDA events around each launch on the context stream).
 * kinds: 0 templates, 1 prep, 2 correlation, 3 harmonic sum + search (device
 * ms); 4 host work until the last launch is queued, 5 host sort + replay,
 * 6 wait for the device and hit read-back (host wall ms, ab_search only),
 * 7 dedispersion (device ms, ab_dedisperse). */
int ab_ctx_set_profiling(ab_ctx *ctx, int on);
int ab_ctx_kernel_times(ab_ctx *ctx, double *ms, long long *launches, int nkinds);
int ab_ctx_reset_kernel_times(ab_ctx *ctx);
long long ab_ctx_launch_count(ab_ctx *ctx);

/* Measured FP32 FMA throughput of this device (TFLOP/s), the denominator of
 * the correlation kernel's roofline: 8 independent FMA chains per thread over
 * 8 CTAs of 256 threads per SM, best of 5 timed runs. */
int ab_measure_fp32_peak(ab_ctx *ctx, double *tflops);

#ifdef __cplusplus
}
#endif
#endif
