// ab_kernels.h -- device-side structures and launch wrappers shared by the
// kernel file and the engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ab_host.h"

namespace ab {

// Read-only per-search constants passed by value to every kernel.
struct SearchConsts {
    double obs_zlo, obs_wlo, obs_rlo;
    long long obs_lobin, numbins;
    long long rlen;            // in-memory plane row length (floats)
    long long clip_col;        // pre-pass blocks write only columns < clip_col
    int corr_uselen, rstep, numz, numws, stages, inmem, nbanks;
    float nph;
    float powcut[AB_MAX_STAGES];
    unsigned *err;             // device error word for bounded waits; may be null
    int superblocks;           // standard search: banks with sbm > 1 share transforms
    const double *norms;       // [block][bank] normalisations (superblock banks)
    int norm_type;             // 0: block median, 1: local power (-locpow)
};

// Blocks of one launch: global ordinal block0 + i, start frequency startr[i].
struct BlockBatch {
    const double *startr;      // device array [nblk]
    long long block0;          // key ordinal of item 0
    int nblk;
    int is_pre;                // pre-pass blocks (in-memory mode only)
};

struct CorrItem {              // one CTA of the correlation kernel
    int bi, bank, t0, nt;
};

struct SigmaConsts {
    double numindep[AB_MAX_STAGES];
};

struct HitBuf {
    unsigned long long *keys;
    float *pows;
    unsigned int *count;
    unsigned int cap;
};

// kernel set (a): templates
void launch_twiddle64(double2 *tw, int n, int sign, cudaStream_t st);
cudaError_t launch_templates(const ab_bank *bank, float2 *bank_out, const double2 *tw_place,
                             const double2 *tw_chirp_all, int chirp_max_log2,
                             double2 *scratch, size_t scratch_elems, cudaStream_t st);
cudaError_t launch_response(double roffset, int numbetween, double z, double w, int numkern,
                            float2 *out, const double2 *tw_chirp_all, int chirp_max_log2,
                            double2 *scratch, cudaStream_t st);

// kernel set (b): spectrum preparation and correlation.  bidx (device, room
// for nbanks ints): banks of one transform length go out in one launch,
// listed there; NULL: one launch per bank (no upload)
cudaError_t launch_prep(const ab_bank *banks_dev, const ab_bank *banks_host, int nbanks,
                        const SearchConsts &sc, const BlockBatch &bb, const float2 *fft,
                        float2 *xhat, long long xhat_per_block, int *bidx, cudaStream_t st);
// per-block normalisations of the superblock banks among banks_host[0..nbanks)
// into sc.norms[block * sc.nbanks + bank index], in one launch listing them in
// bidx (device, room for nbanks ints)
cudaError_t launch_norms(const ab_bank *banks_dev, const ab_bank *banks_host, int nbanks,
                         const SearchConsts &sc, const BlockBatch &bb, const float2 *fft,
                         int *bidx, cudaStream_t st);
// transform units (superblocks, or blocks) of a bank in a batch of nblk blocks
inline int corr_units(const ab_bank &b, const SearchConsts &sc, int nblk)
{
    return (sc.superblocks && b.sbm > 1) ? (nblk + b.sbm - 1) / b.sbm : nblk;
}
cudaError_t launch_corr(int L, const ab_bank *banks_dev, const SearchConsts &sc,
                        const BlockBatch &bb, const CorrItem *items, int nitems,
                        const float2 *xhat, long long xhat_per_block, const float2 *tmpl,
                        float *planes, long long plane_per_block, float *fullplane,
                        cudaStream_t st);

// kernel sets (c)+(d): harmonic summing fused with the threshold search
cudaError_t launch_harmsum_std(const ab_bank *banks_dev, const SearchConsts &sc,
                               const BlockBatch &bb, const float *planes,
                               long long plane_per_block, HitBuf hb, float *dbg,
                               int dbg_bi, cudaStream_t st);
cudaError_t launch_harmsum_inmem(const SearchConsts &sc, const BlockBatch &bb,
                                 const float *fullplane, HitBuf hb, float *dbg, int dbg_bi,
                                 cudaStream_t st);

cudaError_t launch_sigma(HitBuf hb, float *sig, const SigmaConsts &c, cudaStream_t st);

// per-function drop-in helpers
cudaError_t launch_add_ffdot(float *fund, const float *sub, int numws, int numzs, int numrs,
                             int sub_numzs, int sub_numrs, double f, int fund_wlo, int sub_wlo,
                             double fullrlo, long long sub_rlo, double obs_zlo, int sub_zlo,
                             cudaStream_t st);
cudaError_t launch_inmem_add(float *fund, const float *plane, long long rlen, int numzs,
                             int numrs, int fund_rlo, int fund_zlo, double f, cudaStream_t st);
cudaError_t launch_threshold(const float *pw, int numws, int numzs, int numrs, float powcut,
                             int stage, HitBuf hb, cudaStream_t st);

cudaError_t launch_fma_peak(float *out, int iters, int sms, cudaStream_t st);
cudaError_t launch_tc_gemm(const float *A, const float *B, float *C, int N, int K, int split,
                           unsigned *err, cudaStream_t st);

// kernel set (b'), tensor-core correlation: the banded template product as a
// complex contraction in split BF16 or FP16 (hi + lo) with FP32 accumulation.
constexpr int TC_TILE_T = 128;          // templates per tile (MMA N = 2 per template)
constexpr int TC_ATILE = 128;           // output positions per accumulator (MMA M)
constexpr int TC_ACC = 1;               // accumulators (128 x 256 FP32, 256 TMEM columns) per CTA
constexpr int TC_STAGES = 3;            // template K-step ring
constexpr int TC_CHUNK = 64 * 2 * TC_TILE_T;   // bytes of one K step (hi + lo) at N = 256

struct TcTile {                 // templates perm[t0 .. t0+nt) of one bank
    int bank, t0, nt, n;        // n = MMA N = 2 nt rounded up to 16
    int c_lo, nks;              // first tap (multiple of 8) and K steps of 8 taps
    long long off;              // byte offset of the packed operand (parity 0;
                                // parity 1 follows after nks * 64 n bytes)
};
struct TcItem {                 // one CTA: positions a0 .. a0 + 128 TC_ACC - 1 of one parity
    int bi, tile, parity, a0;
};

cudaError_t launch_tc_raw(const ab_bank *b, int stride, float2 *out, const double2 *tw_all,
                          int max_log2, cudaStream_t st);
cudaError_t launch_tc_pack(const ab_bank *b, const TcTile *tiles_dev, int ntiles, int nks_max,
                           const int *perm_dev, const float2 *raw, int stride,
                           unsigned char *pack, int fp16, cudaStream_t st);
cudaError_t launch_prep_time(const ab_bank *banks_dev, const ab_bank *banks_host, int nbanks,
                             const SearchConsts &sc, const BlockBatch &bb, const float2 *fft,
                             float2 *dtime, long long dt_per_block, cudaStream_t st);
cudaError_t launch_corr_tc(const ab_bank *banks_dev, const SearchConsts &sc, const BlockBatch &bb,
                           const TcItem *items, int nitems, const TcTile *tiles, const int *perm,
                           const float2 *dtime, long long dt_per_block, const unsigned char *pack,
                           int nks_max, float *planes, long long plane_per_block, float *fullplane,
                           int fp16, cudaStream_t st);
size_t tc_corr_smem(int nks_max);

// candidate polishing (optimize_accelcand for acceleration searches)
struct PolishIn {
    double r, z;
    int numharm;
    int mode;                   // 0: max_rz_arr_harmonics, 1: max_rz_arr (one harmonic)
};
cudaError_t launch_polish(const float2 *data, long long numdata, long long lobin, const PolishIn *in,
                          int n, ab_polished *out, cudaStream_t st);

// Jerk-search polishing: one job = one response (gen_z_response or
// gen_w_response at roffset, numbetween nb, numkern points) and the
// correlation outputs that use it, out_j[o] giving output o's offset j:
//   amp[o] = sum_i d[beginbin + i] conj(resp[nb i - j]),  0 <= nb i - j < numkern,
// d = 0 outside the spectrum.  mode 2 copies bin beginbin (rz_interp's exact
// bin case).
constexpr int RZW_PMAX = 4096;              // largest in-shared-memory FFT of a chirp phase
constexpr int RZW_NMAX_LOG2 = 17;           // chirps up to 2^17 samples
constexpr int RZW_VOL = 17 * 17 * 24;       // (w, z, r) cells of one harmonic's volume
struct RzwJob {
    double roffset, z, w;
    long long beginbin;
    long long resp_off;                     // float2 offset of the response in the scratch
    long long acc_off;                      // double2 offset of the accumulator (npts > RZW_PMAX)
    int mode;                               // 0: z response, 1: w response, 2: copy a bin
    int nb, numkern, npts;
    int nout, out_off;                      // amplitudes out_amp[out_off .. + nout)
    int j_off;                              // their correlation offsets out_j[j_off .. + nout),
                                            // shared by the jobs of one volume
};
cudaError_t launch_rzw_jobs(const RzwJob *jobs, int njobs, const float2 *data, long long numdata,
                            const double2 *tw, float2 *resp, double2 *acc, const long long *out_j,
                            float2 *out_amp, cudaStream_t st);
// Per candidate c: harmonics' local powers from the amplitudes
// amp[lp_off[c * 32 + h] ...] (lp_n of them; mean over NUMLOCPOWAVG = 20;
// lp_n < 0: 1, raw powers), the float sum over harmonics of |vol|^2 / locpow
// in the reference's order (volume amplitudes at amp[vol_off[c] + h * ncell +
// cell]) and the first cell of the highest sum: best[c] = cell index,
// bestval[c] (if not null) = that sum.
cudaError_t launch_rzw_sum(const float2 *amp, const int *numharm, const int *vol_off,
                           const int *lp_off, const int *lp_n, int ncell, int ncand, int *best,
                           float *bestval, cudaStream_t st);
// max_rzw_arr_harmonics for every candidate (host planning + the two
// kernels above): data is the device spectrum of numdata bins, tw the FP64
// table exp(-2 pi i m / 2^RZW_NMAX_LOG2), budget the response scratch per
// launch.  Returns an AB_* code, with a message in err on failure.
int rzw_optimize(const float2 *data, long long numdata, long long lobin, const ab_cand *cands,
                 long long n, ab_polished *out, const double2 *tw, size_t budget, cudaStream_t st,
                 char *err, size_t errlen, long long *launches);
// -noharmpolish: max_rzw_arr (src/maximize_rzw.c:3-52) for every harmonic
// of every candidate, each on its own.
int rzw_optimize_each(const float2 *data, long long numdata, long long lobin, const ab_cand *cands,
                      long long n, ab_polished *out, const double2 *tw, size_t budget,
                      cudaStream_t st, char *err, size_t errlen, long long *launches);

// subband dedispersion (prepsubband): x time-major [nspec][nchan] ->
// D [nsub][dedisp_sub_pitch(nspec / ds)] -> out [ndm][nspec / ds]; maxcd the
// largest channel delay; off the subband offsets on the device, off_host the
// same on the host (the DM stage's window sizes are chosen from them)
long long dedisp_sub_pitch(long long nout);
cudaError_t launch_dedisp(const float *x, long long nspec, int nchan, const int *cd, int maxcd,
                          int nsub, int ds, const int *off, const int *off_host, int ndm, float *D,
                          float *out, cudaStream_t st);

// time-series input path: realfft and deredden
constexpr int AB_DERED_MAXW = 1024;     // longest de-reddening block
bool realfft_supported(long long n);
bool pow2_fft_supported(long long M);
long long bluestein_len(long long M);
cudaError_t launch_realfft(const float *series, float2 *out, float2 *scratch, long long n, cudaStream_t st);
// any even n (1024 <= n <= 2^26): a: bluestein_len(n/2) points of work, scratch
// as many, B the cached transform of the chirp kernel (rebuilt when build_B)
cudaError_t launch_realfft_bluestein(const float *series, float2 *out, float2 *a, float2 *scratch,
                                     float2 *B, bool build_B, long long n, cudaStream_t st);
cudaError_t launch_deredden(float2 *fft, const int2 *blocks, int nb, float *means, cudaStream_t st);

}  // namespace ab
