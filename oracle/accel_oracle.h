/*
 * accel_oracle.h -- CPU restatement of PRESTO's accelsearch hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This oracle is the checker for the CUDA
 * engine in presto_b200/: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load it.  Nothing
 * in the product links against it.
 *
 * Each function restates the reference algorithm (PRESTO 6.0.1) and cites
 * the reference file:line it follows.  The library is built twice from the
 * same source (oracle/Makefile):
 *   liboracle64.so  ORC_REAL=double -- the FP64 oracle used for parity
 *   liboracle32.so  ORC_REAL=float  -- FP32 arithmetic like the reference's
 *                                      FFTW single-precision path; used as
 *                                      the timed CPU baseline
 *
 * Pinning: the response generators are pinned to the reference's own
 * known-answer tests (tests/test_presto_python.py:117-146), the Fresnel
 * integrals to the reference's fresnl.c compiled from its sources into
 * oracle/_ref/, and the GSL-boundary statistics to scipy.special.  The full
 * reference path needs FFTW3f, GSL and glib, which are absent, so it is not
 * built; plane-level parity is therefore anchored on this restatement.
 */
#ifndef ACCEL_ORACLE_H
#define ACCEL_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { float r, i; } orc_fcomplex;          /* include/ransomfft.h:13-16 */

/* Search options that reach the hot path (clig/accelsearch_cmd.cli). */
typedef struct {
    long long N;          /* samples in the time series (.inf N) */
    double dt;            /* sample time (s) */
    long long numbins;    /* complex bins in the .fft file */
    int zmax, wmax, wmaxP;
    int numharm;
    float sigma;
    double flo, fhi; int floP, fhiP;
    double rlo, rhi; int rloP, rhiP;
    long long lobin;
    int inmemP;
    float nph;            /* >0: photon normalisation (-photon) */
    int locpowP;          /* -locpow: local-power normalisation */
    int noharmpolishP;    /* -noharmpolish */
} orc_params;

/* Geometry subset of accelobs (include/accel.h:37-81). */
typedef struct {
    long long N, numbins, lobin, highestbin;
    int maxkernlen, corr_uselen, fftlen, numharmstages, numz, numw;
    int numbetween, inmem, norm_type, rstep;
    double dt, T, rlo, rhi, dr, zlo, zhi, dz, wlo, whi, dw;
    float nph, sigma;
    float powcut[6];
    long long numindep[6];
    int noharmpolish;             /* 1: -noharmpolish (src/accel_utils.c:1489-1494) */
} orc_obs;

/* One plane (ffdotpows, include/accel.h:120-130), powers[w][z][r]. */
typedef struct {
    long long rlo;
    int zlo, wlo, numrs, numzs, numws;
    float *powers;
    unsigned short *rinds, *zinds;     /* borrowed from the bank */
} orc_ffdot;

typedef struct orc_bank orc_bank;      /* subharminfo + its kernels */

typedef struct {
    float power, sigma;
    int numharm;
    double r, z, w;
} orc_cand;

typedef struct {
    long long block;      /* block ordinal in the main loop */
    int stage, wi, zi, ri;
    float power;
} orc_hit;

/* ---- geometry ---- */
int  orc_next_good_fftlen(int n);
int  orc_fftlen_from_kernwidth(int kernwidth);
int  orc_z_resp_halfwidth(double z);
int  orc_w_resp_halfwidth(double z, double w);
int  orc_calc_required_z(double harm_fract, double zfull);
int  orc_calc_required_w(double harm_fract, double wfull);
double orc_calc_required_r(double harm_fract, double rfull);
int  orc_obs_init(const orc_params *p, orc_obs *obs);

/* ---- statistics ---- */
double orc_chi2_logp(double chi2, double dof);
double orc_equivalent_gaussian_sigma(double logp);
double orc_candidate_sigma(double power, int numsum, double numtrials);
double orc_power_for_sigma(double sigma, int numsum, double numtrials);
double orc_gauss_q(double x);
double orc_gauss_qinv(double q);
double orc_chisq_q(double chi2, double dof);
double orc_chisq_qinv(double q, double dof);
float  orc_median(float *arr, int n);

/* ---- responses ---- */
void orc_fresnel(double x, double *s, double *c);
int  orc_gen_r_response(double roffset, int numbetween, int numkern, orc_fcomplex *out);
int  orc_gen_z_response(double roffset, int numbetween, double z, int numkern, orc_fcomplex *out);
int  orc_gen_w_response(double roffset, int numbetween, double z, double w, int numkern,
                        orc_fcomplex *out);

/* ---- FFT (unnormalised, sign -1 forward / +1 inverse) ---- */
void orc_cfft_double(double *data, int n, int sign);

/* ---- engine ---- */
orc_bank *orc_bank_create(const orc_obs *obs, int numharm, int harmnum);
void      orc_bank_free(orc_bank *b);
int       orc_bank_info(const orc_bank *b, int *zmax, int *wmax, int *numkern_zdim,
                        int *numkern_wdim, int *fftlen, int *halfwidth);
int       orc_bank_kernel(const orc_bank *b, int wi, int zi, orc_fcomplex *out);

int  orc_subharm_fderivs_vol(const orc_obs *obs, const orc_fcomplex *fft, int numharm,
                             int harmnum, double fullrlo, double fullrhi, orc_bank *bank,
                             orc_ffdot *out);
void orc_ffdot_free(orc_ffdot *f);
void orc_add_ffdotpows(orc_ffdot *fund, const orc_ffdot *sub, int numharm, int harmnum);
void orc_fund_to_ffdotplane(const orc_ffdot *ffd, const orc_obs *obs, float *plane);
void orc_inmem_add_ffdotpows(orc_ffdot *fund, const orc_obs *obs, const float *plane,
                             int numharm, int harmnum);

/* Full search (src/accelsearch.c:161-224).  Hits are recorded in visit
 * order when hits != NULL.  max_blocks < 0 means all blocks; otherwise only
 * blocks [first_block, first_block + max_blocks) of the main loop are
 * searched (bounded CPU samples).  Returns number of candidates or < 0. */
void orc_last_timing(double *setup_s, double *blocks_s);
/* Thread-seconds the last search's block loop spent in its correlation FFTs
 * (forward and inverse) and the loop's wall time x threads. */
void orc_last_fft_share(double *fft_thread_s, double *loop_thread_s);
/* Threads of later searches' block loops (0: the template banks' count), so
 * that a one-thread block loop can be timed without one-thread banks. */
void orc_set_loop_threads(int n);
/* The same search over every block_stride-th block from first_block
 * (max_blocks of them; a CPU sample spread over the spectrum).  In-memory
 * searches ignore the stride. */
long long orc_accelsearch_sample(const orc_params *p, const orc_fcomplex *fft, int nthreads,
                                 long long first_block, long long max_blocks,
                                 long long block_stride, orc_cand *cands, long long maxcands,
                                 orc_hit *hits, long long maxhits, long long *numhits,
                                 long long *numblocks_done);
long long orc_accelsearch(const orc_params *p, const orc_fcomplex *fft, int nthreads,
                          long long first_block, long long max_blocks,
                          orc_cand *cands, long long maxcands,
                          orc_hit *hits, long long maxhits, long long *numhits,
                          long long *numblocks_done);

/* Candidate list replay (src/accel_utils.c:387-469 and :1412-1452). */
typedef struct orc_list orc_list;
orc_list *orc_list_new(void);
void      orc_list_free(orc_list *l);
int       orc_list_insert(orc_list *l, float power, float sigma, int numharm,
                          double rr, double zz, double ww);
long long orc_list_get(const orc_list *l, orc_cand *out, long long maxout);
void      orc_search_ffdotpows(const orc_ffdot *ffd, int numharm, const orc_obs *obs,
                               orc_list *l, long long block, orc_hit *hits,
                               long long maxhits, long long *numhits);

/* ---- candidate polishing (polish_oracle.c) ---------------------------- */
#define ORC_MAX_HARM 32
typedef struct {                 /* rderivs, include/presto.h:160-168 */
    double pow, phs, dpow, dphs, d2pow, d2phs, locpow;
} orc_rderivs;
typedef struct {                 /* fourierprops, include/presto.h:170-188 */
    double r;
    float rerr;
    double z;
    float zerr;
    double w;
    float werr;
    float pow, powerr, sig, rawpow, phs, phserr, cen, cenerr, pur, purerr, locpow;
} orc_fourierprops;

int    orc_z_resp_halfwidth_acc(double z, int highacc);
int    orc_w_resp_halfwidth_acc(double z, double w, int highacc);
void   orc_rzw_interp(const orc_fcomplex *data, long numdata, double r, double z, double w,
                      int kern_half_width, orc_fcomplex *ans);
double orc_get_localpower3d(const orc_fcomplex *data, long numdata, double r, double z, double w);
void   orc_get_derivs3d(const orc_fcomplex *data, long numdata, double r, double z, double w,
                        double localpower, orc_rderivs *res);
int    orc_calc_props(const orc_rderivs *d, double r, double z, double w, orc_fourierprops *o);
typedef struct {                 /* rzwerrs, include/presto.h:233-246 */
    double p, pd, pdd, f, fd, fdd;
    float perr, pderr, pdderr, ferr, fderr, fdderr;
} orc_rzwerrs;
int    orc_calc_rzwerrs(const orc_fourierprops *p, double T, orc_rzwerrs *o);
double orc_max_rz_arr(const orc_fcomplex *data, long numdata, double rin, double zin,
                      double *rout, double *zout, orc_rderivs *derivs);
void   orc_max_rz_arr_harmonics(const orc_fcomplex *data, long numdata, int numharm, double rin,
                                double zin, double *rout, double *zout, orc_rderivs *derivs,
                                double *powers);
int    orc_optimize_accelcand(const orc_fcomplex *fft, long long numbins, long long lobin,
                              int numharm, double r, double z, double *pows, double *hirs,
                              double *hizs, orc_rderivs *derivs);
int    orc_optimize_cands(const orc_fcomplex *fft, long long numbins, long long lobin, int ncand,
                          const int *numharm, const double *r, const double *z, double *pows,
                          double *hirs, double *hizs, orc_rderivs *derivs, int nthreads);
/* jerk searches (numw > 0): max_rzw_arr / max_rzw_arr_harmonics */
void   orc_rzw_vol_point(const orc_fcomplex *data, long numdata, long beginbin, int numbetween,
                         long j, const orc_fcomplex *resp, int numkern, orc_fcomplex *out);
double orc_max_rzw_arr(const orc_fcomplex *data, long numdata, double rin, double zin, double win,
                       double *rout, double *zout, double *wout, orc_rderivs *derivs);
void   orc_max_rzw_arr_harmonics(const orc_fcomplex *data, long numdata, int numharm, double rin,
                                 double zin, double win, double *rout, double *zout, double *wout,
                                 orc_rderivs *derivs, double *powers);
int    orc_optimize_cands_w(const orc_fcomplex *fft, long long numbins, long long lobin, int ncand,
                            int jerk, const int *numharm, const double *r, const double *z,
                            const double *w, double *pows, double *hirs, double *hizs,
                            double *hiws, orc_rderivs *derivs, int nthreads);

/* ---- time-series input path (series_oracle.c) -------------------------- */
int   orc_realfft_forward(float *data, long n);
float orc_invsqrtf(float x);
void  orc_loc_pow(const float *pw, int n, float *local);
long  orc_deredden(orc_fcomplex *fft, long numbins, int startwidth, int endwidth, double endfreq,
                   double T);

#ifdef __cplusplus
}
#endif
#endif
