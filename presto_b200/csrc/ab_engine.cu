// ab_engine.cu -- device orchestration behind the C ABI of accel_b200.h:
// context and memory management, the template-bank cache, block batching of
// the whole-spectrum search, the per-function drop-ins, and kernel timing.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "ab_host.h"
#include "ab_index.h"
#include "ab_kernels.h"

using namespace ab;

namespace {

constexpr int kTwLog2 = 14;                 // FP64 twiddle table for FFTs up to 16384
constexpr int kNumKinds = 8;   // templates, prep, corr, harmsum (device); host setup, host replay,
                               // hit fetch; dedispersion (device)
double now_ms()
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <typename T> struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    cudaError_t ensure(size_t want)
    {
        if (want <= n) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc(&p, want * sizeof(T));
        if (e == cudaSuccess) n = want;
        return e;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

}  // namespace

struct ab_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    size_t hbm_budget = 0;
    size_t scratch_budget = 8ull << 30;

    // template banks
    ab_bankset bs{};
    bool have_banks = false;
    // template banks: entries of the device-wide cache (shared by every
    // context on the device); tmpl_p points into the current one
    // operands of the tensor-core correlation for one bank set: templates
    // sorted by half-width into tiles, packed split-BF16 taps per tile
    struct TcBank {
        bool ready = false;                 // tiles and permutation
        std::vector<TcTile> tiles;          // bank-major
        std::vector<int> tile_lo;           // first tile of each bank, nbanks + 1 entries
        DevBuf<TcTile> dtiles;
        DevBuf<int> dperm;
        DevBuf<unsigned char> pack[2];      // packed operands: split BF16, split FP16
        bool pack_ready[2] = {false, false};
        long long pack_bytes = 0;
        int nks_max = 0;
    };
    struct BankEntry {
        ab_bankset bs;
        DevBuf<float2> tmpl;
        unsigned long long used = 0;
        TcBank tc;
        int refs = 0;                       // contexts whose current banks these are
        cudaEvent_t ready = nullptr;        // templates written (recorded by the builder)
    };
    BankEntry *cur_bank = nullptr;
    int corr_path = AB_CORR_FFT;            // correlation path of searches and drop-ins
    DevBuf<float2> dtime;                   // normalised block data (tensor-core path)
    DevBuf<float2> ser_in, ser_scr;         // time-series input path
    DevBuf<float2> blu_a, blu_b;            // Bluestein work and chirp-kernel transform
    DevBuf<float> dd_x, dd_sub, dd_out;     // dedispersion: spectra, subbands, DM trials
    DevBuf<float2> dd_fft;                  // spectrum of one DM trial (ab_search_dedispersed)
    DevBuf<int> bidx;                       // bank lists of the grouped preparation launches
    DevBuf<int> dd_cd, dd_off;              // dedispersion delays
    long long blu_M = 0;                    // the length blu_b was built for
    DevBuf<int2> dered_blocks;
    DevBuf<float> dered_means;
    DevBuf<TcItem> titems;
    float2 *tmpl_p = nullptr;
    DevBuf<ab_bank> dbanks;
    DevBuf<double2> tw64;
    DevBuf<double2> tw_rzw;                 // exp(-2 pi i m / 2^RZW_NMAX_LOG2), jerk polishing
    DevBuf<float2> resp;

    // spectrum, scratch, planes
    DevBuf<float2> fft;
    long long fft_bins = 0;
    bool fft_valid = false;
    DevBuf<float2> xhat;
    DevBuf<double> norms;                    // [block][bank] of superblock banks
    DevBuf<float> planes;
    DevBuf<float> fullplane;
    DevBuf<double> startr;
    DevBuf<CorrItem> items;
    DevBuf<float> dbg;
    DevBuf<float> tmpa, tmpb;
    DevBuf<unsigned> errw;                   // device error word

    // hits: a ring of kHitSets sets, so that the device runs up to
    // kHitSets - 1 batches ahead of the host's replay (batches that hold a
    // strong signal cross the threshold millions of times and replay slowly);
    // set 0 is keys/pows/sigs/count, set i > 0 the (i - 1)th of the _x arrays
    static constexpr int kHitSets = 4;
    DevBuf<unsigned long long> keys, keys_x[kHitSets - 1];
    DevBuf<float> pows, pows_x[kHitSets - 1];
    DevBuf<unsigned int> count, count_x[kHitSets - 1];
    DevBuf<float> sigs, sigs_x[kHitSets - 1];
    std::vector<float> hsigs;
    unsigned *hcount = nullptr;              // pinned [kHitSets]
    // pinned staging of large uploads from pageable host memory (h2d_staged)
    static constexpr size_t kStage = (size_t) 64 << 20;
    char *stage[2] = {nullptr, nullptr};
    cudaEvent_t stage_done[2] = {};
    cudaEvent_t batch_done[kHitSets] = {};
    cudaStream_t cstream = nullptr;          // device->host copies of hits
    unsigned int hit_cap = 1u << 22;
    std::vector<unsigned long long> hkeys;
    std::vector<float> hpows;
    std::vector<double> hstart;
    std::vector<ab_cand> last_cands;
    int worklog_on = 0;                 // record the .txtcand lines of each ab_search
    std::string last_worklog;
    unsigned overflow_need = 0;              // hits one batch wanted beyond hit_cap
    bool hits_truncated = false;             // host copy holds only the latest batches

    // timing
    bool prof = false;
    double kms[kNumKinds] = {0, 0, 0, 0, 0, 0, 0, 0};
    long long kn[kNumKinds] = {0, 0, 0, 0, 0, 0, 0, 0};
    long long launches = 0;
    std::vector<cudaEvent_t> evpool;
    std::vector<std::pair<int, int>> evpending;   // (kind, event index)
    int evused = 0;
};

static int fail(ab_ctx *c, int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

#define CK(call)                                                                             \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail(ctx, AB_ERR_CUDA, "%s failed: %s (%s:%d)", #call,                    \
                        cudaGetErrorString(e_), __FILE__, __LINE__);                         \
    } while (0)

// ---- timing helpers -------------------------------------------------------
static void tick(ab_ctx *ctx, int kind, bool begin)
{
    if (!ctx->prof) return;
    if (ctx->evused >= (int) ctx->evpool.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        ctx->evpool.push_back(e);
    }
    int idx = ctx->evused++;
    cudaEventRecord(ctx->evpool[idx], ctx->stream);
    if (!begin) ctx->evpending.push_back({kind, idx});
}

static void harvest(ab_ctx *ctx)
{
    if (!ctx->prof) return;
    cudaStreamSynchronize(ctx->stream);
    for (auto &pe : ctx->evpending) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->evpool[pe.second - 1], ctx->evpool[pe.second]);
        ctx->kms[pe.first] += ms;
        ctx->kn[pe.first] += 1;
    }
    ctx->evpending.clear();
    ctx->evused = 0;
}

// ---- banks ----------------------------------------------------------------
// Template banks are shared by every context of a device: a request pool's
// workers and plain contexts reuse the banks any of them built.  Entries are
// reference-counted by the contexts whose current banks they are; a cache
// miss builds into an unreferenced entry (least recently used, once the cache
// holds kBankCache) after a device synchronisation, so no queued kernel of
// any stream still reads it.  The builder records an event that later users
// wait on.  Every search and drop-in returns with its stream drained, so a
// context that moves to other banks leaves nothing in flight on the old ones.
constexpr int kBankCache = 16;
constexpr int kMaxDevices = 64;

struct SharedBanks {
    std::mutex mu;
    std::vector<ab_ctx::BankEntry *> entries;
    unsigned long long clock = 0;
    int live = 0;                           // contexts alive on the device
};
static SharedBanks g_banks[kMaxDevices];

static void free_entry(ab_ctx::BankEntry *e)
{
    e->tmpl.release();
    e->tc.dtiles.release();
    e->tc.dperm.release();
    e->tc.pack[0].release();
    e->tc.pack[1].release();
    if (e->ready) cudaEventDestroy(e->ready);
    delete e;
}

static bool same_templates(const ab_bankset &a, const ab_bankset &b)
{
    if (a.nbanks != b.nbanks) return false;
    for (int i = 0; i < a.nbanks; i++) {
        const ab_bank &x = a.b[i], &y = b.b[i];
        if (x.numharm != y.numharm || x.harmnum != y.harmnum || x.zmax != y.zmax ||
            x.wmax != y.wmax || x.L != y.L)
            return false;
    }
    return true;
}

// The context's FP64 twiddle table, used by every response and template
// transform; built on first use, since a context whose banks come from the
// device-wide cache never generates templates itself.
static int ensure_tw64(ab_ctx *ctx)
{
    if (ctx->tw64.n) return AB_OK;
    CK(ctx->tw64.ensure((size_t) 1 << (kTwLog2 - 1)));
    launch_twiddle64(ctx->tw64.p, 1 << kTwLog2, -1, ctx->stream);
    CK(cudaGetLastError());
    return AB_OK;
}

// Makes the template banks of obs current: from the device-wide cache when a
// search with the same template geometry ran before, else built on the device.
static int ensure_banks(ab_ctx *ctx, const ab_obs *obs)
{
    ab_bankset nb;
    int rc = ab_bankset_init(obs, &nb);
    if (rc) return fail(ctx, rc, "unsupported search geometry (FFT span above 4096 or "
                                 "circular wrap into valid cells)");
    CK(ctx->dbanks.ensure(AB_MAX_BANKS));
    SharedBanks &sb = g_banks[ctx->device];
    std::lock_guard<std::mutex> lock(sb.mu);
    ab_ctx::BankEntry *hit = nullptr;
    for (auto *e : sb.entries)
        if (e->bs.nbanks && same_templates(e->bs, nb)) hit = e;
    if (hit) {
        CK(cudaStreamWaitEvent(ctx->stream, hit->ready, 0));
    } else {
        if (int rc2 = ensure_tw64(ctx)) return rc2;
        ab_ctx::BankEntry *victim = nullptr;
        if ((int) sb.entries.size() >= kBankCache)
            for (auto *e : sb.entries)
                if (e->refs == 0 && e != ctx->cur_bank && (!victim || e->used < victim->used)) victim = e;
        if (victim) {
            CK(cudaDeviceSynchronize());    // nothing queued may still read it
            hit = victim;
        } else {
            hit = new ab_ctx::BankEntry();
            sb.entries.push_back(hit);
        }
        hit->bs.nbanks = 0;
        hit->tc.ready = false;                  // a reused entry's operands are stale
        hit->tc.pack_ready[0] = hit->tc.pack_ready[1] = false;
        if (!hit->ready) CK(cudaEventCreateWithFlags(&hit->ready, cudaEventDisableTiming));
        CK(hit->tmpl.ensure((size_t) nb.tmpl_total));
        for (int i = 0; i < nb.nbanks; i++) {
            tick(ctx, 0, true);
            cudaError_t e = launch_templates(&nb.b[i], hit->tmpl.p + nb.b[i].tmpl_off, nullptr,
                                             ctx->tw64.p, kTwLog2, nullptr, 0, ctx->stream);
            tick(ctx, 0, false);
            ctx->launches++;
            if (e != cudaSuccess)
                return fail(ctx, AB_ERR_CUDA, "template generation failed: %s", cudaGetErrorString(e));
        }
        CK(cudaEventRecord(hit->ready, ctx->stream));
        hit->bs = nb;
    }
    if (ctx->cur_bank != hit) {
        if (ctx->cur_bank) ctx->cur_bank->refs--;
        hit->refs++;
    }
    hit->used = ++sb.clock;
    ctx->tmpl_p = hit->tmpl.p;
    ctx->cur_bank = hit;
    ctx->bs = nb;
    ctx->have_banks = true;
    CK(cudaMemcpyAsync(ctx->dbanks.p, nb.b, sizeof(ab_bank) * nb.nbanks, cudaMemcpyHostToDevice,
                       ctx->stream));
    return AB_OK;
}

static SearchConsts make_consts(const ab_obs *obs, const ab_bankset &bs)
{
    SearchConsts sc{};
    sc.obs_zlo = obs->zlo;
    sc.obs_wlo = obs->wlo;
    sc.obs_rlo = obs->rlo;
    sc.obs_lobin = obs->lobin;
    sc.numbins = obs->numbins;
    sc.rlen = (obs->highestbin + obs->corr_uselen) * (long long) AB_RDR;
    sc.clip_col = (long long) obs->rlo * AB_RDR;
    sc.corr_uselen = obs->corr_uselen;
    sc.rstep = obs->rstep;
    sc.numz = obs->numz;
    sc.numws = obs->numw > 0 ? obs->numw : 1;
    sc.stages = obs->numharmstages;
    sc.inmem = obs->inmem;
    sc.nbanks = bs.nbanks;
    sc.nph = obs->nph;
    sc.norm_type = obs->norm_type;
    for (int i = 0; i < AB_MAX_STAGES; i++) sc.powcut[i] = i < obs->numharmstages ? obs->powcut[i] : 0.f;
    sc.err = nullptr;
    return sc;
}

// Correlation work items of one batch of nblk blocks, grouped by FFT length.
struct CorrPlan {
    std::vector<CorrItem> items;
    int Ls[8];
    int off[8], cnt[8];
    int nL = 0;
};

// With sc.superblocks, a bank of superblock height m > 1 has one transform
// unit per m consecutive blocks of the batch (CorrItem.bi is the unit).
static void build_corr_plan(const ab_bankset &bs, const SearchConsts &sc, int nblk, int bank_lo,
                            int bank_hi, CorrPlan &p)
{
    p.items.clear();
    p.nL = 0;
    for (int L = 512; L <= 8192; L <<= 1) {
        int start = (int) p.items.size();
        const int G = L >= 4096 ? 1 : 4096 / L, tile = 16 * G;
        for (int k = bank_lo; k < bank_hi; k++) {
            const ab_bank &b = bs.b[k];
            if (b.L != L) continue;
            const int units = corr_units(b, sc, nblk);
            for (int t0 = 0; t0 < b.ntmpl; t0 += tile)
                for (int bi = 0; bi < units; bi++)
                    p.items.push_back(CorrItem{bi, k, t0, std::min(tile, b.ntmpl - t0)});
        }
        int n = (int) p.items.size() - start;
        if (n > 0) {
            p.Ls[p.nL] = L;
            p.off[p.nL] = start;
            p.cnt[p.nL] = n;
            p.nL++;
        }
    }
}

static int run_corr(ab_ctx *ctx, const SearchConsts &sc, const BlockBatch &bb, const CorrPlan &p,
                    const CorrItem *ditems, float *planes, long long ppb, float *fullplane)
{
    for (int i = 0; i < p.nL; i++) {
        tick(ctx, 2, true);
        cudaError_t e = launch_corr(p.Ls[i], ctx->dbanks.p, sc, bb, ditems + p.off[i], p.cnt[i],
                                    ctx->xhat.p, ctx->bs.xhat_per_block, ctx->tmpl_p, planes,
                                    ppb, fullplane, ctx->stream);
        tick(ctx, 2, false);
        ctx->launches++;
        if (e != cudaSuccess)
            return fail(ctx, AB_ERR_CUDA, "correlation launch failed: %s", cudaGetErrorString(e));
    }
    return AB_OK;
}

static int run_prep(ab_ctx *ctx, const SearchConsts &sc, const BlockBatch &bb, const float2 *fft,
                    int bank_lo, int bank_hi)
{
    tick(ctx, 1, true);
    CK(ctx->bidx.ensure((size_t) std::max(1, bank_hi - bank_lo)));
    cudaError_t e = launch_prep(ctx->dbanks.p + bank_lo, ctx->bs.b + bank_lo, bank_hi - bank_lo,
                                sc, bb, fft, ctx->xhat.p, ctx->bs.xhat_per_block, ctx->bidx.p,
                                ctx->stream);
    tick(ctx, 1, false);
    {
        // one launch per distinct transform length
        unsigned seen = 0;
        for (int k = bank_lo; k < bank_hi; k++) seen |= 1u << (31 - __builtin_clz((unsigned) ctx->bs.b[k].L));
        ctx->launches += __builtin_popcount(seen);
    }
    if (e != cudaSuccess)
        return fail(ctx, AB_ERR_CUDA, "prep launch failed: %s", cudaGetErrorString(e));
    return AB_OK;
}

// ---- tensor-core correlation ---------------------------------------------
// Tiles of the current bank set: per bank, templates sorted by half-width
// (widest first, then by index) in groups of TC_TILE_T, each covering the taps
// [hw0 - hwmax, hw0 + hwmax) of its widest member rounded out to 8; then the
// raw responses and the packed split operand (BF16 or FP16), built once per
// bank set and format.
static int tc_fmt(const ab_ctx *ctx) { return ctx->corr_path == AB_CORR_TC_SPLIT_FP16 ? 1 : 0; }

// Tiles and template permutation of the current bank set (shared by both
// 16-bit formats); the caller holds the bank lock.
static int ensure_tc_tiles(ab_ctx *ctx, ab_ctx::TcBank &tb)
{
    if (tb.ready) return AB_OK;
    const ab_bankset &bs = ctx->bs;
    tb.tiles.clear();
    tb.tile_lo.assign(1, 0);
    std::vector<int> perm;
    long long off = 0;
    int nks_max = 0;
    for (int k = 0; k < bs.nbanks; k++) {
        const ab_bank &b = bs.b[k];
        std::vector<int> hw(b.ntmpl), order(b.ntmpl);
        for (int t = 0; t < b.ntmpl; t++) {
            int wi = t / b.nz, zi = t - wi * b.nz;
            hw[t] = ab_w_resp_halfwidth((double) (-b.zmax + zi * AB_DZ), (double) (-b.wmax + wi * AB_DW));
            order[t] = t;
        }
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return hw[x] > hw[y]; });
        const int pbase = (int) perm.size();
        perm.insert(perm.end(), order.begin(), order.end());
        for (int i0 = 0; i0 < b.ntmpl; i0 += TC_TILE_T) {
            TcTile t{};
            t.bank = k;
            t.t0 = pbase + i0;
            t.nt = std::min(TC_TILE_T, b.ntmpl - i0);
            t.n = (2 * t.nt + 15) / 16 * 16;
            const int hwmax = hw[order[i0]];
            t.c_lo = (b.hw0 - hwmax) / 8 * 8;
            const int c_hi = (b.hw0 + hwmax + 7) / 8 * 8;
            t.nks = (c_hi - t.c_lo) / 8;
            t.off = off;
            off += 2LL * t.nks * 64 * t.n;
            nks_max = std::max(nks_max, t.nks);
            tb.tiles.push_back(t);
        }
        tb.tile_lo.push_back((int) tb.tiles.size());
    }
    if (tc_corr_smem(nks_max) > 227 * 1024)
        return fail(ctx, AB_ERR_ARG, "template responses too wide for the tensor-core path");
    CK(tb.dtiles.ensure(tb.tiles.size()));
    CK(tb.dperm.ensure(perm.size()));
    CK(cudaMemcpyAsync(tb.dtiles.p, tb.tiles.data(), sizeof(TcTile) * tb.tiles.size(),
                       cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(tb.dperm.p, perm.data(), sizeof(int) * perm.size(), cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));           // perm is a host vector
    tb.pack_bytes = off;
    tb.nks_max = nks_max;
    tb.ready = true;
    return AB_OK;
}

// The raw responses and the packed operand of the context's 16-bit format,
// built once per bank set and format.
static int ensure_tc(ab_ctx *ctx)
{
    // the operands live in the shared bank entry: built under its lock
    std::lock_guard<std::mutex> lock(g_banks[ctx->device].mu);
    ab_ctx::TcBank &tb = ctx->cur_bank->tc;
    const int fmt = tc_fmt(ctx);
    if (tb.ready && tb.pack_ready[fmt]) return AB_OK;
    if (int rc0 = ensure_tw64(ctx)) return rc0;
    if (int rc0 = ensure_tc_tiles(ctx, tb)) return rc0;
    const ab_bankset &bs = ctx->bs;
    CK(tb.pack[fmt].ensure((size_t) tb.pack_bytes));
    DevBuf<float2> raw;
    int ntmax = 0, stride_max = 0;
    for (int k = 0; k < bs.nbanks; k++) {
        ntmax = std::max(ntmax, bs.b[k].ntmpl);
        stride_max = std::max(stride_max, 4 * bs.b[k].hw0);
    }
    CK(raw.ensure((size_t) ntmax * stride_max));
    int rc = AB_OK;
    for (int k = 0; k < bs.nbanks && rc == AB_OK; k++) {
        const ab_bank &b = bs.b[k];
        const int lo = tb.tile_lo[k], nt = tb.tile_lo[k + 1] - lo;
        int nks_k = 0;
        for (int i = lo; i < lo + nt; i++) nks_k = std::max(nks_k, tb.tiles[i].nks);
        tick(ctx, 0, true);
        cudaError_t e = launch_tc_raw(&b, 4 * b.hw0, raw.p, ctx->tw64.p, kTwLog2, ctx->stream);
        if (e == cudaSuccess)
            e = launch_tc_pack(&b, tb.dtiles.p + lo, nt, nks_k, tb.dperm.p, raw.p, 4 * b.hw0,
                               tb.pack[fmt].p, fmt, ctx->stream);
        tick(ctx, 0, false);
        ctx->launches += 2;
        if (e != cudaSuccess)
            rc = fail(ctx, AB_ERR_CUDA, "tensor-core operand packing failed: %s", cudaGetErrorString(e));
    }
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    raw.release();
    if (rc) return rc;
    if (e != cudaSuccess)
        return fail(ctx, AB_ERR_CUDA, "tensor-core operand packing failed: %s", cudaGetErrorString(e));
    tb.pack_ready[fmt] = true;
    return AB_OK;
}

// Work items of one batch of nblk blocks over banks [bank_lo, bank_hi):
// longest tiles first; the blocks of one (tile, parity, positions) are
// adjacent so that they share the tile's operand in L2.
static void build_tc_plan(const ab_ctx::TcBank &tb, const ab_bankset &bs, int nblk, int bank_lo,
                          int bank_hi, std::vector<TcItem> &items)
{
    items.clear();
    std::vector<int> order;
    for (int i = tb.tile_lo[bank_lo]; i < tb.tile_lo[bank_hi]; i++) order.push_back(i);
    std::stable_sort(order.begin(), order.end(),
                     [&](int x, int y) { return tb.tiles[x].nks > tb.tiles[y].nks; });
    for (int i : order) {
        const ab_bank &b = bs.b[tb.tiles[i].bank];
        for (int p = 0; p < 2; p++) {
            const int na = (b.numrs_max - p + 1) / 2;
            for (int a0 = 0; a0 < na; a0 += TC_ACC * TC_ATILE)
                for (int bi = 0; bi < nblk; bi++) items.push_back(TcItem{bi, i, p, a0});
        }
    }
}

// Normalised data and tensor-core correlation of one batch.
static int run_tc(ab_ctx *ctx, const SearchConsts &sc, const BlockBatch &bb, const float2 *fft,
                  int bank_lo, int bank_hi, const TcItem *ditems, int nitems, float *planes,
                  long long ppb, float *fullplane)
{
    const ab_ctx::TcBank &tb = ctx->cur_bank->tc;
    tick(ctx, 1, true);
    cudaError_t e = launch_prep_time(ctx->dbanks.p + bank_lo, ctx->bs.b + bank_lo, bank_hi - bank_lo,
                                     sc, bb, fft, ctx->dtime.p, ctx->bs.dtime_per_block, ctx->stream);
    tick(ctx, 1, false);
    ctx->launches++;
    if (e != cudaSuccess) return fail(ctx, AB_ERR_CUDA, "data preparation failed: %s", cudaGetErrorString(e));
    tick(ctx, 2, true);
    const int fmt = tc_fmt(ctx);
    e = launch_corr_tc(ctx->dbanks.p, sc, bb, ditems, nitems, tb.dtiles.p, tb.dperm.p, ctx->dtime.p,
                       ctx->bs.dtime_per_block, tb.pack[fmt].p, tb.nks_max, planes, ppb, fullplane,
                       fmt, ctx->stream);
    tick(ctx, 2, false);
    ctx->launches++;
    if (e != cudaSuccess)
        return fail(ctx, AB_ERR_CUDA, "tensor-core correlation launch failed: %s", cudaGetErrorString(e));
    return AB_OK;
}

// Hit set i of the context (0 or 1).
struct HitSet {
    unsigned long long *keys;
    float *pows, *sigs;
    unsigned *count;
};

static int ensure_hitsets(ab_ctx *ctx)
{
    CK(ctx->keys.ensure(ctx->hit_cap));
    CK(ctx->pows.ensure(ctx->hit_cap));
    CK(ctx->sigs.ensure(ctx->hit_cap));
    CK(ctx->count.ensure(1));
    for (int i = 0; i < ab_ctx::kHitSets - 1; i++) {
        CK(ctx->keys_x[i].ensure(ctx->hit_cap));
        CK(ctx->pows_x[i].ensure(ctx->hit_cap));
        CK(ctx->sigs_x[i].ensure(ctx->hit_cap));
        CK(ctx->count_x[i].ensure(1));
    }
    if (!ctx->hcount)
        CK(cudaHostAlloc((void **) &ctx->hcount, ab_ctx::kHitSets * sizeof(unsigned),
                         cudaHostAllocDefault));
    for (int i = 0; i < ab_ctx::kHitSets; i++)
        if (!ctx->batch_done[i]) CK(cudaEventCreateWithFlags(&ctx->batch_done[i], cudaEventDisableTiming));
    if (!ctx->cstream) CK(cudaStreamCreateWithFlags(&ctx->cstream, cudaStreamNonBlocking));
    return AB_OK;
}

static HitSet hitset(ab_ctx *ctx, int i)
{
    if (i == 0) return HitSet{ctx->keys.p, ctx->pows.p, ctx->sigs.p, ctx->count.p};
    return HitSet{ctx->keys_x[i - 1].p, ctx->pows_x[i - 1].p, ctx->sigs_x[i - 1].p,
                  ctx->count_x[i - 1].p};
}

// After the launches that fill hit set i: sigma of every hit, the count to
// pinned host memory, and an event marking the set complete.
static int close_hitset(ab_ctx *ctx, const ab_obs *obs, int i)
{
    HitSet h = hitset(ctx, i);
    SigmaConsts c{};
    for (int k = 0; k < AB_MAX_STAGES; k++)
        c.numindep[k] = k < obs->numharmstages ? (double) obs->numindep[k] : 1.0;
    HitBuf hb{h.keys, h.pows, h.count, ctx->hit_cap};
    CK(launch_sigma(hb, h.sigs, c, ctx->stream));
    ctx->launches++;
    CK(cudaMemcpyAsync(ctx->hcount + i, h.count, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaEventRecord(ctx->batch_done[i], ctx->stream));
    return AB_OK;
}

// Replays the batches' threshold crossings into the candidate list on a
// thread of its own, batch after batch in the order they are handed over (the
// reference's visit order), while the search keeps launching batches: the
// device never waits for the list.  The worker alone writes the list and the
// context's host copy of the hits until finish() has joined it.
struct Replayer {
    struct Batch {
        std::vector<unsigned long long> keys;
        std::vector<float> pows, sigs;
    };
    ab_ctx *ctx;
    const ab_obs *obs;
    ab_list *list;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Batch> q;
    bool closing = false;
    int rc = AB_OK;
    double ms = 0.0;
    std::thread th;

    Replayer(ab_ctx *c, const ab_obs *o, ab_list *l) : ctx(c), obs(o), list(l)
    {
        th = std::thread([this] { run(); });
    }
    ~Replayer() { finish(); }
    void push(Batch &&b)
    {
        {
            std::lock_guard<std::mutex> lock(mu);
            q.push_back(std::move(b));
        }
        cv.notify_one();
    }
    int finish()
    {
        {
            std::lock_guard<std::mutex> lock(mu);
            closing = true;
        }
        cv.notify_one();
        if (th.joinable()) th.join();
        return rc;
    }
    void run()
    {
        for (;;) {
            Batch b;
            {
                std::unique_lock<std::mutex> lock(mu);
                cv.wait(lock, [this] { return closing || !q.empty(); });
                if (q.empty()) return;
                b = std::move(q.front());
                q.pop_front();
            }
            const long long n = (long long) b.keys.size();
            if (rc == AB_OK) {
                const double t0 = now_ms();
                const int r = ab_replay_hits(obs, b.keys.data(), b.pows.data(), b.sigs.data(), n,
                                             ctx->hstart.data(), ab_num_blocks(obs), list);
                ms += now_ms() - t0;
                if (r) rc = r;
            }
            keep_hits(ctx, b.keys, b.pows, b.sigs);
        }
    }
    // the context's copy of the search's hits (ab_last_hits); bounded: past
    // 2^24 only the latest batches are kept.  The batch's vectors are taken
    // over when the copy is empty (the common case: one batch holds them all).
    static void keep_hits(ab_ctx *ctx, std::vector<unsigned long long> &k, std::vector<float> &p,
                          std::vector<float> &sg)
    {
        if (ctx->hkeys.size() + k.size() > (size_t) 1 << 24) {
            ctx->hkeys.clear();
            ctx->hpows.clear();
            ctx->hsigs.clear();
            ctx->hits_truncated = true;
        }
        if (ctx->hkeys.empty()) {
            ctx->hkeys.swap(k);
            ctx->hpows.swap(p);
            ctx->hsigs.swap(sg);
            return;
        }
        ctx->hkeys.insert(ctx->hkeys.end(), k.begin(), k.end());
        ctx->hpows.insert(ctx->hpows.end(), p.begin(), p.end());
        ctx->hsigs.insert(ctx->hsigs.end(), sg.begin(), sg.end());
    }
};

// Waits for hit set i and copies its hits to the host, freeing the set for
// the next batch; hands them to the replayer (or, without a list, keeps them).
static int drain_hitset(ab_ctx *ctx, int i, Replayer *rp)
{
    CK(cudaEventSynchronize(ctx->batch_done[i]));
    unsigned n = ctx->hcount[i];
    if (n > ctx->hit_cap) {
        ctx->overflow_need = n;
        return fail(ctx, AB_ERR_OVERFLOW, "%u threshold crossings in one batch exceed the hit "
                                          "buffer (%u)", n, ctx->hit_cap);
    }
    if (n == 0) return AB_OK;
    HitSet h = hitset(ctx, i);
    Replayer::Batch b;
    b.keys.resize(n);
    b.pows.resize(n);
    b.sigs.resize(n);
    CK(cudaMemcpyAsync(b.keys.data(), h.keys, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost,
                       ctx->cstream));
    CK(cudaMemcpyAsync(b.pows.data(), h.pows, sizeof(float) * n, cudaMemcpyDeviceToHost, ctx->cstream));
    CK(cudaMemcpyAsync(b.sigs.data(), h.sigs, sizeof(float) * n, cudaMemcpyDeviceToHost, ctx->cstream));
    CK(cudaStreamSynchronize(ctx->cstream));
    if (rp) rp->push(std::move(b));
    else Replayer::keep_hits(ctx, b.keys, b.pows, b.sigs);
    return AB_OK;
}

// Core search over main-loop blocks [first, first+count).  All hits are kept
// in ctx->hkeys/hpows/hsigs; with list != NULL they are also replayed into
// the candidate list, batch by batch while the device computes the next
// batch.  dbg_block >= 0 dumps that block's stage sums into ctx->dbg.
static int search_core(ab_ctx *ctx, const ab_obs *obs, const float2 *dfft, long long first,
                       long long count, long long dbg_block, ab_list *list,
                       double *replay_ms = nullptr)
{
    const ab_bankset &bs = ctx->bs;
    SearchConsts sc = make_consts(obs, bs);
    CK(ctx->errw.ensure(1));
    CK(cudaMemsetAsync(ctx->errw.p, 0, sizeof(unsigned), ctx->stream));
    sc.err = ctx->errw.p;
    long long nmain = ab_num_blocks(obs), npre = ab_num_preblocks(obs);
    if (first < 0) first = 0;
    if (count < 0 || first + count > nmain) count = nmain - first;
    if (count < 0) count = 0;
    if (nmain >= (1ll << AB_KEY_BBITS) || sc.numz >= (1 << AB_KEY_ZBITS) ||
        sc.numws >= (1 << AB_KEY_WBITS) || obs->corr_uselen >= (1 << AB_KEY_RBITS))
        return fail(ctx, AB_ERR_ARG, "search too large for the hit key layout");
    ctx->hstart.resize((size_t) (nmain + npre + 1));
    ab_block_starts(obs, ctx->hstart.data(), nmain);
    ab_preblock_starts(obs, ctx->hstart.data() + nmain, npre);
    CK(ctx->startr.ensure(ctx->hstart.size()));
    CK(cudaMemcpyAsync(ctx->startr.p, ctx->hstart.data(), sizeof(double) * (nmain + npre),
                       cudaMemcpyHostToDevice, ctx->stream));
    int rc = ensure_hitsets(ctx);
    if (rc) return rc;
    ctx->hkeys.clear();
    ctx->hpows.clear();
    ctx->hsigs.clear();
    ctx->hits_truncated = false;
    // with a list: the replay runs on its own thread (joined on every return)
    std::unique_ptr<Replayer> rp(list ? new Replayer(ctx, obs, list) : nullptr);
    auto finish_replay = [&]() -> int {
        if (!rp) return AB_OK;
        const int r = rp->finish();
        if (replay_ms) *replay_ms += rp->ms;
        if (r) return fail(ctx, r, "hit replay failed");
        return AB_OK;
    };
    const int nstage = obs->numharmstages;
    const size_t dbg_floats = (size_t) nstage * sc.numws * sc.numz * obs->corr_uselen;
    if (dbg_block >= 0) CK(ctx->dbg.ensure(dbg_floats));

    if (obs->inmem) {
        // full plane: every block (pre-pass and main loop) is correlated into
        // it; sums read rows of lower frequency, so the whole plane comes first
        long long nall = nmain + npre;
        size_t rows = (size_t) sc.numz * sc.rlen;
        CK(ctx->fullplane.ensure(rows));
        long long first_col = 2 * (long long) (npre > 0 ? 8.0 : obs->rlo);
        if (first_col > sc.rlen) first_col = sc.rlen;
        if (first_col > 0)
            CK(cudaMemset2DAsync(ctx->fullplane.p, sizeof(float) * sc.rlen, 0,
                                 sizeof(float) * first_col, sc.numz, ctx->stream));
        const bool tcp = ctx->corr_path != AB_CORR_FFT;
        if (tcp) {
            rc = ensure_tc(ctx);
            if (rc) return rc;
            CK(ctx->dtime.ensure((size_t) std::max<long long>(std::max(npre, nmain), 1) *
                                 bs.dtime_per_block));
        } else {
            CK(ctx->xhat.ensure((size_t) std::max<long long>(nall, 1) * bs.xhat_per_block));
        }
        // both passes' work items are built first and uploaded once, each pass
        // reading its own part, so the passes follow each other on the stream
        CorrPlan plan[2];
        std::vector<TcItem> tplan[2];
        size_t ioff[2] = {0, 0}, itotal = 0;
        for (int pass = 0; pass < 2; pass++) {
            const long long nb = pass == 0 ? npre : nmain;
            ioff[pass] = itotal;
            if (nb == 0) continue;
            if (tcp) {
                build_tc_plan(ctx->cur_bank->tc, bs, (int) nb, 0, 1, tplan[pass]);
                itotal += tplan[pass].size();
            } else {
                build_corr_plan(bs, sc, (int) nb, 0, 1, plan[pass]);
                itotal += plan[pass].items.size();
            }
        }
        if (tcp) {
            CK(ctx->titems.ensure(std::max<size_t>(itotal, 1)));
            for (int pass = 0; pass < 2; pass++)
                if (!tplan[pass].empty())
                    CK(cudaMemcpyAsync(ctx->titems.p + ioff[pass], tplan[pass].data(),
                                       sizeof(TcItem) * tplan[pass].size(), cudaMemcpyHostToDevice,
                                       ctx->stream));
        } else {
            CK(ctx->items.ensure(std::max<size_t>(itotal, 1)));
            for (int pass = 0; pass < 2; pass++)
                if (!plan[pass].items.empty())
                    CK(cudaMemcpyAsync(ctx->items.p + ioff[pass], plan[pass].items.data(),
                                       sizeof(CorrItem) * plan[pass].items.size(),
                                       cudaMemcpyHostToDevice, ctx->stream));
        }
        for (int pass = 0; pass < 2; pass++) {
            long long nb = pass == 0 ? npre : nmain;
            if (nb == 0) continue;
            BlockBatch bb{ctx->startr.p + (pass == 0 ? nmain : 0), 0, (int) nb, pass == 0};
            if (tcp) {
                rc = run_tc(ctx, sc, bb, dfft, 0, 1, ctx->titems.p + ioff[pass], (int) tplan[pass].size(),
                            nullptr, 0, ctx->fullplane.p);
                if (rc) return rc;
                continue;
            }
            rc = run_prep(ctx, sc, bb, dfft, 0, 1);
            if (rc) return rc;
            rc = run_corr(ctx, sc, bb, plan[pass], ctx->items.p + ioff[pass], nullptr, 0,
                          ctx->fullplane.p);
            if (rc) return rc;
        }
        // the sums run in chunks of blocks through the ring of hit sets, so the
        // host replays chunk k while the device sums the chunks after it
        const long long nch = std::min<long long>(8, std::max<long long>(1, count / 32));
        const long long csz = (count + nch - 1) / nch;
        int k = 0;
        for (long long c0 = first; count > 0 && c0 < first + count; c0 += csz, k++) {
            const int nb = (int) std::min<long long>(csz, first + count - c0);
            const int set = k % ab_ctx::kHitSets;
            HitSet h = hitset(ctx, set);
            CK(cudaMemsetAsync(h.count, 0, sizeof(unsigned), ctx->stream));
            BlockBatch bb{ctx->startr.p + c0, c0, nb, 0};
            HitBuf hb{h.keys, h.pows, h.count, ctx->hit_cap};
            const bool dump = dbg_block >= c0 && dbg_block < c0 + nb;
            tick(ctx, 3, true);
            cudaError_t e = launch_harmsum_inmem(sc, bb, ctx->fullplane.p, hb,
                                                 dump ? ctx->dbg.p : nullptr,
                                                 dump ? (int) (dbg_block - c0) : -1, ctx->stream);
            tick(ctx, 3, false);
            ctx->launches++;
            if (e != cudaSuccess)
                return fail(ctx, AB_ERR_CUDA, "harmonic sum launch failed: %s", cudaGetErrorString(e));
            rc = close_hitset(ctx, obs, set);
            if (rc) return rc;
            if (k >= ab_ctx::kHitSets - 1) {
                rc = drain_hitset(ctx, (k - (ab_ctx::kHitSets - 1)) % ab_ctx::kHitSets, rp.get());
                if (rc) return rc;
            }
        }
        for (int d = std::max(0, k - (ab_ctx::kHitSets - 1)); d < k; d++) {
            rc = drain_hitset(ctx, d % ab_ctx::kHitSets, rp.get());
            if (rc) return rc;
        }
        return finish_replay();
    }

    // standard mode: batches of blocks, each correlated for every bank, then
    // summed; hit sets rotate so the host replays batch k - (kHitSets - 1)
    // meanwhile
    const bool tcp = ctx->corr_path != AB_CORR_FFT;
    if (tcp) {
        rc = ensure_tc(ctx);
        if (rc) return rc;
    }
    const size_t per_block = (size_t) bs.plane_per_block * sizeof(float) +
                             (size_t) (tcp ? bs.dtime_per_block : bs.xhat_per_block) * sizeof(float2);
    long long B = (long long) (ctx->scratch_budget / std::max<size_t>(per_block, 1));
    if (B < 1) B = 1;
    if (B > 512) B = 512;
    // several batches per search let the replay overlap the device work
    if (count >= 8 && B > (count + 7) / 8) B = (count + 7) / 8;
    if (B > count) B = std::max<long long>(count, 1);
    CK(ctx->planes.ensure((size_t) B * bs.plane_per_block));
    CorrPlan full, tail;
    std::vector<TcItem> tfull, ttail;
    long long rem = count % B;
    if (tcp) {
        CK(ctx->dtime.ensure((size_t) B * bs.dtime_per_block));
        build_tc_plan(ctx->cur_bank->tc, bs, (int) B, 0, bs.nbanks, tfull);
        if (rem) build_tc_plan(ctx->cur_bank->tc, bs, (int) rem, 0, bs.nbanks, ttail);
        CK(ctx->titems.ensure(tfull.size() + ttail.size()));
        CK(cudaMemcpyAsync(ctx->titems.p, tfull.data(), sizeof(TcItem) * tfull.size(),
                           cudaMemcpyHostToDevice, ctx->stream));
        if (rem)
            CK(cudaMemcpyAsync(ctx->titems.p + tfull.size(), ttail.data(), sizeof(TcItem) * ttail.size(),
                               cudaMemcpyHostToDevice, ctx->stream));
    } else {
        CK(ctx->xhat.ensure((size_t) B * bs.xhat_per_block));
        sc.superblocks = 1;
        CK(ctx->norms.ensure((size_t) B * bs.nbanks));
        sc.norms = ctx->norms.p;
        build_corr_plan(bs, sc, (int) B, 0, bs.nbanks, full);
        if (rem) build_corr_plan(bs, sc, (int) rem, 0, bs.nbanks, tail);
        CK(ctx->items.ensure(full.items.size() + tail.items.size()));
        CK(cudaMemcpyAsync(ctx->items.p, full.items.data(), sizeof(CorrItem) * full.items.size(),
                           cudaMemcpyHostToDevice, ctx->stream));
        if (rem)
            CK(cudaMemcpyAsync(ctx->items.p + full.items.size(), tail.items.data(),
                               sizeof(CorrItem) * tail.items.size(), cudaMemcpyHostToDevice, ctx->stream));
    }
    int k = 0;
    for (long long b0 = first; b0 < first + count; b0 += B, k++) {
        int nb = (int) std::min<long long>(B, first + count - b0);
        const int set = k % ab_ctx::kHitSets;
        HitSet h = hitset(ctx, set);
        CK(cudaMemsetAsync(h.count, 0, sizeof(unsigned), ctx->stream));
        BlockBatch bb{ctx->startr.p + b0, b0, nb, 0};
        if (tcp) {
            const TcItem *di = ctx->titems.p + ((nb == B) ? 0 : tfull.size());
            const int ni = (int) ((nb == B) ? tfull.size() : ttail.size());
            rc = run_tc(ctx, sc, bb, dfft, 0, bs.nbanks, di, ni, ctx->planes.p, bs.plane_per_block,
                        nullptr);
            if (rc) return rc;
        } else {
            tick(ctx, 1, true);
            CK(ctx->bidx.ensure((size_t) std::max(1, bs.nbanks)));
            cudaError_t en = launch_norms(ctx->dbanks.p, bs.b, bs.nbanks, sc, bb, dfft, ctx->bidx.p,
                                          ctx->stream);
            tick(ctx, 1, false);
            ctx->launches++;
            if (en != cudaSuccess)
                return fail(ctx, AB_ERR_CUDA, "normalisation launch failed: %s", cudaGetErrorString(en));
            rc = run_prep(ctx, sc, bb, dfft, 0, bs.nbanks);
            if (rc) return rc;
            const CorrPlan &p = (nb == B) ? full : tail;
            const CorrItem *di = ctx->items.p + ((nb == B) ? 0 : full.items.size());
            rc = run_corr(ctx, sc, bb, p, di, ctx->planes.p, bs.plane_per_block, nullptr);
            if (rc) return rc;
        }
        int dbi = (dbg_block >= b0 && dbg_block < b0 + nb) ? (int) (dbg_block - b0) : -1;
        HitBuf hb{h.keys, h.pows, h.count, ctx->hit_cap};
        tick(ctx, 3, true);
        cudaError_t e = launch_harmsum_std(ctx->dbanks.p, sc, bb, ctx->planes.p, bs.plane_per_block,
                                           hb, dbi >= 0 ? ctx->dbg.p : nullptr, dbi, ctx->stream);
        tick(ctx, 3, false);
        ctx->launches++;
        if (e != cudaSuccess)
            return fail(ctx, AB_ERR_CUDA, "harmonic sum launch failed: %s", cudaGetErrorString(e));
        rc = close_hitset(ctx, obs, set);
        if (rc) return rc;
        if (k >= ab_ctx::kHitSets - 1) {
            rc = drain_hitset(ctx, (k - (ab_ctx::kHitSets - 1)) % ab_ctx::kHitSets, rp.get());
            if (rc) return rc;
        }
    }
    for (int d = std::max(0, k - (ab_ctx::kHitSets - 1)); d < k; d++) {
        rc = drain_hitset(ctx, d % ab_ctx::kHitSets, rp.get());
        if (rc) return rc;
    }
    return finish_replay();
}

static int fetch_hits(ab_ctx *ctx, long long *nhits)
{
    unsigned n = 0;
    CK(cudaMemcpyAsync(&n, ctx->count.p, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (n > ctx->hit_cap) {
        ctx->hkeys.clear();
        ctx->hpows.clear();
        return fail(ctx, AB_ERR_OVERFLOW, "%u threshold crossings exceed the hit buffer (%u)", n,
                    ctx->hit_cap);
    }
    ctx->hkeys.resize(n);
    ctx->hpows.resize(n);
    if (n) {
        CK(cudaMemcpyAsync(ctx->hkeys.data(), ctx->keys.p, sizeof(unsigned long long) * n,
                           cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(ctx->hpows.data(), ctx->pows.p, sizeof(float) * n, cudaMemcpyDeviceToHost,
                           ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    *nhits = n;
    return AB_OK;
}

// Device-side failures that do not abort a kernel (a bounded wait that ran
// out) are reported through the context's error word.
static int check_device_error(ab_ctx *ctx)
{
    unsigned e = 0;
    if (!ctx->errw.p) return AB_OK;
    CK(cudaMemcpyAsync(&e, ctx->errw.p, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (e) return fail(ctx, AB_ERR_CUDA, "device wait timed out (error word 0x%x)", e);
    return AB_OK;
}

// Device arrays of float2 (complex spectra, series read in pairs) must be
// 8-byte aligned; a misaligned pointer is refused instead of faulting.
static bool misaligned8(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 7u) != 0; }

// Upload of `bytes` from pageable host memory on the context's stream.  A
// pageable copy is staged by the driver on one host thread (~11 GB/s); copies
// of 256 MB or more (filterbank spectra) go instead through two pinned
// buffers that several host threads fill in parallel, each buffer's transfer
// overlapping the filling of the other.  The call returns when the source has
// been read.
static int h2d_staged(ab_ctx *ctx, void *dst, const void *src, size_t bytes)
{
    const size_t chunk = ab_ctx::kStage;
    if (bytes < 4 * chunk) {
        CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
        return AB_OK;
    }
    for (int i = 0; i < 2; i++) {
        if (!ctx->stage[i]) CK(cudaHostAlloc((void **) &ctx->stage[i], chunk, cudaHostAllocDefault));
        if (!ctx->stage_done[i])
            CK(cudaEventCreateWithFlags(&ctx->stage_done[i], cudaEventDisableTiming));
    }
    const unsigned hw = std::thread::hardware_concurrency();
    const int nthr = (int) std::max(1u, std::min(8u, hw / 2));
    const char *s = static_cast<const char *>(src);
    char *d = static_cast<char *>(dst);
    size_t off = 0;
    for (int k = 0; off < bytes; k++) {
        const size_t n = std::min(chunk, bytes - off);
        char *buf = ctx->stage[k & 1];
        // the buffer's last transfer (of this call or an earlier one) is done
        CK(cudaEventSynchronize(ctx->stage_done[k & 1]));
        std::vector<std::thread> th;
        int started = 1;
        try {
            for (int t = 1; t < nthr; t++, started++)
                th.emplace_back([=] {
                    const size_t a = n * t / nthr, b = n * (t + 1) / nthr;
                    memcpy(buf + a, s + off + a, b - a);
                });
        } catch (...) {                 // no thread: this one copies the rest
        }
        memcpy(buf, s + off, n / nthr);
        if (started < nthr)
            memcpy(buf + n * started / nthr, s + off + n * started / nthr, n - n * started / nthr);
        for (auto &x : th) x.join();
        CK(cudaMemcpyAsync(d + off, buf, n, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaEventRecord(ctx->stage_done[k & 1], ctx->stream));
        off += n;
    }
    return AB_OK;
}

static int use_device(ab_ctx *ctx)
{
    CK(cudaSetDevice(ctx->device));
    return AB_OK;
}

// ============================================================================
// C ABI
// ============================================================================
extern "C" {

int ab_ctx_create(int device, ab_ctx **out)
{
    if (!out) return AB_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0 ||
        device >= kMaxDevices)
        return AB_ERR_CUDA;
    ab_ctx *ctx = new ab_ctx();
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return AB_ERR_CUDA;
    }
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    ctx->hbm_budget = (size_t) (0.85 * (double) fr);
    ctx->scratch_budget = std::min<size_t>(8ull << 30, ctx->hbm_budget / 4);
    {
        std::lock_guard<std::mutex> lock(g_banks[device].mu);
        g_banks[device].live++;
    }
    *out = ctx;
    return AB_OK;
}

void ab_ctx_destroy(ab_ctx *ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    {
        SharedBanks &sb = g_banks[ctx->device];
        std::lock_guard<std::mutex> lock(sb.mu);
        if (ctx->cur_bank) ctx->cur_bank->refs--;
        ctx->cur_bank = nullptr;
        if (--sb.live == 0) {
            // the last context on the device: the cache goes with it
            for (auto *e : sb.entries) free_entry(e);
            sb.entries.clear();
        }
    }
    ctx->dbanks.release();
    ctx->tw64.release();
    ctx->tw_rzw.release();
    ctx->resp.release();
    ctx->fft.release();
    ctx->xhat.release();
    ctx->planes.release();
    ctx->fullplane.release();
    ctx->startr.release();
    ctx->items.release();
    ctx->dbg.release();
    ctx->tmpa.release();
    ctx->tmpb.release();
    ctx->errw.release();
    ctx->dtime.release();
    ctx->ser_in.release();
    ctx->ser_scr.release();
    ctx->blu_a.release();
    ctx->blu_b.release();
    ctx->blu_M = 0;
    ctx->dd_x.release();
    ctx->dd_sub.release();
    ctx->dd_out.release();
    ctx->dd_fft.release();
    ctx->bidx.release();
    ctx->dd_cd.release();
    ctx->dd_off.release();
    ctx->dered_blocks.release();
    ctx->dered_means.release();
    ctx->titems.release();
    ctx->norms.release();
    ctx->keys.release();
    ctx->pows.release();
    ctx->count.release();
    ctx->sigs.release();
    for (int i = 0; i < ab_ctx::kHitSets - 1; i++) {
        ctx->keys_x[i].release();
        ctx->pows_x[i].release();
        ctx->count_x[i].release();
        ctx->sigs_x[i].release();
    }
    if (ctx->hcount) cudaFreeHost(ctx->hcount);
    for (int i = 0; i < 2; i++) {
        if (ctx->stage[i]) cudaFreeHost(ctx->stage[i]);
        if (ctx->stage_done[i]) cudaEventDestroy(ctx->stage_done[i]);
    }
    for (int i = 0; i < ab_ctx::kHitSets; i++)
        if (ctx->batch_done[i]) cudaEventDestroy(ctx->batch_done[i]);
    if (ctx->cstream) cudaStreamDestroy(ctx->cstream);
    for (auto e : ctx->evpool) cudaEventDestroy(e);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char *ab_ctx_last_error(const ab_ctx *ctx) { return ctx ? ctx->err.c_str() : "no context"; }

void *ab_ctx_stream(ab_ctx *ctx) { return ctx ? (void *) ctx->stream : nullptr; }

// Correlation cost per template and transform at each device FFT length from
// 512 to 4096: a fundamental-like bank of 128 templates (half-width L/16,
// 3L/4 valid columns) over 148 blocks, k_corr timed with CUDA events (best of
// 3 after a warm-up) on zeroed data.  The table replaces the process-wide one.
int ab_autotune(ab_ctx *ctx, double *costs_out, int n)
{
    if (!ctx || n < 0) return AB_ERR_ARG;
    int rc = use_device(ctx);
    if (rc) return rc;
    constexpr int kBlocks = 148, kTmpl = 128, kLmax = 4096;
    DevBuf<float2> xhat, tmpl;
    DevBuf<float> planes;
    DevBuf<double> startr;
    DevBuf<ab_bank> dbank;
    DevBuf<CorrItem> items;
    auto release = [&]() {
        xhat.release();
        tmpl.release();
        planes.release();
        startr.release();
        dbank.release();
        items.release();
    };
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double costs[AB_COST_SLOTS] = {0};
    cudaError_t e = cudaSuccess;
    do {
        if ((e = xhat.ensure((size_t) kBlocks * kLmax / 2)) != cudaSuccess) break;
        if ((e = tmpl.ensure((size_t) kTmpl * kLmax)) != cudaSuccess) break;
        if ((e = planes.ensure((size_t) kBlocks * kTmpl * (kLmax * 3 / 4))) != cudaSuccess) break;
        if ((e = startr.ensure(kBlocks)) != cudaSuccess) break;
        if ((e = dbank.ensure(1)) != cudaSuccess) break;
        if ((e = items.ensure((size_t) kBlocks * kTmpl)) != cudaSuccess) break;
        cudaMemsetAsync(xhat.p, 0, sizeof(float2) * xhat.n, ctx->stream);
        cudaMemsetAsync(tmpl.p, 0, sizeof(float2) * tmpl.n, ctx->stream);
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        for (int L = 512; L <= kLmax && e == cudaSuccess; L <<= 1) {
            ab_bank b{};
            b.numharm = b.harmnum = 1;
            b.f = 1.0;
            b.nz = b.ntmpl = kTmpl;
            b.nw = 1;
            b.fftlen_ref = L;
            b.L = L;
            b.hw0 = L / 16;
            b.numrs_max = 3 * L / 4;
            b.sbm = 1;
            SearchConsts sc{};
            sc.corr_uselen = b.numrs_max;
            sc.rstep = b.numrs_max / 2;
            sc.numz = kTmpl;
            sc.numws = 1;
            sc.nbanks = 1;
            std::vector<double> st(kBlocks);
            for (int k = 0; k < kBlocks; k++) st[k] = 1000.0 + (double) k * sc.rstep;
            const int G = L >= 4096 ? 1 : 4096 / L, tile = 16 * G;
            std::vector<CorrItem> it;
            for (int t0 = 0; t0 < kTmpl; t0 += tile)
                for (int bi = 0; bi < kBlocks; bi++) it.push_back(CorrItem{bi, 0, t0, tile});
            cudaMemcpyAsync(dbank.p, &b, sizeof b, cudaMemcpyHostToDevice, ctx->stream);
            cudaMemcpyAsync(startr.p, st.data(), sizeof(double) * kBlocks, cudaMemcpyHostToDevice,
                            ctx->stream);
            cudaMemcpyAsync(items.p, it.data(), sizeof(CorrItem) * it.size(), cudaMemcpyHostToDevice,
                            ctx->stream);
            BlockBatch bb{startr.p, 0, kBlocks, 0};
            float best = 1e30f;
            for (int rep = 0; rep < 4 && e == cudaSuccess; rep++) {
                cudaEventRecord(e0, ctx->stream);
                e = launch_corr(L, dbank.p, sc, bb, items.p, (int) it.size(), xhat.p, L / 2, tmpl.p,
                                planes.p, (long long) kTmpl * b.numrs_max, nullptr, ctx->stream);
                cudaEventRecord(e1, ctx->stream);
                if (e == cudaSuccess) e = cudaEventSynchronize(e1);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (rep > 0 && ms < best) best = ms;
            }
            int lg = 0;
            while ((1 << lg) < L) lg++;
            costs[lg] = (double) best / ((double) kBlocks * kTmpl);
        }
    } while (0);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaError_t es = cudaStreamSynchronize(ctx->stream);
    release();
    if (e == cudaSuccess) e = es;
    if (e != cudaSuccess) return fail(ctx, AB_ERR_CUDA, "autotune failed: %s", cudaGetErrorString(e));
    ab_set_transform_costs(costs, AB_COST_SLOTS);
    for (int i = 0; i < n && costs_out; i++) costs_out[i] = i < AB_COST_SLOTS ? costs[i] : 0.0;
    return AB_OK;
}

int ab_optimize_cands(ab_ctx *ctx, const ab_obs *obs, const ab_fcomplex *fft, int fft_on_device,
                      const ab_cand *cands, long long n, ab_polished *out)
{
    if (!ctx || !obs || !fft || (n > 0 && (!cands || !out)) || n < 0) return AB_ERR_ARG;
    if (n == 0) return AB_OK;
    if (n > (1 << 24)) return fail(ctx, AB_ERR_ARG, "too many candidates");
    if (fft_on_device && misaligned8(fft))
        return fail(ctx, AB_ERR_ARG, "device spectrum not 8-byte aligned");
    int rc = use_device(ctx);
    if (rc) return rc;
    const float2 *dfft = reinterpret_cast<const float2 *>(fft);
    if (!fft_on_device) {
        CK(ctx->fft.ensure((size_t) obs->numbins));
        CK(cudaMemcpyAsync(ctx->fft.p, fft, sizeof(float2) * obs->numbins, cudaMemcpyHostToDevice,
                           ctx->stream));
        ctx->fft_bins = obs->numbins;
        ctx->fft_valid = true;
        dfft = ctx->fft.p;
    }
    for (long long k = 0; k < n; k++)
        if (cands[k].numharm < 1 || cands[k].numharm > AB_POLISH_MAX_HARM)
            return fail(ctx, AB_ERR_ARG, "candidate %lld has %d harmonics", k, cands[k].numharm);
    if (obs->numw > 0) {
        // jerk search: max_rzw_arr_harmonics (src/accel_utils.c:563-568)
        if (ctx->tw_rzw.n == 0) {
            CK(ctx->tw_rzw.ensure((size_t) 1 << (RZW_NMAX_LOG2 - 1)));
            launch_twiddle64(ctx->tw_rzw.p, 1 << RZW_NMAX_LOG2, -1, ctx->stream);
            CK(cudaGetLastError());
        }
        char msg[256] = {0};
        const size_t budget = std::min<size_t>(ctx->scratch_budget, 1ull << 30);
        // candidates in groups of at most 4096 harmonics bound each plan's host
        // memory (about 7000 volume outputs per harmonic)
        for (long long c0 = 0; c0 < n;) {
            long long c1 = c0, nh = 0;
            while (c1 < n && (c1 == c0 || nh + cands[c1].numharm <= 4096)) nh += cands[c1++].numharm;
            rc = !obs->noharmpolish
                     ? rzw_optimize(dfft, obs->numbins, obs->lobin, cands + c0, c1 - c0, out + c0,
                                    ctx->tw_rzw.p, budget, ctx->stream, msg, sizeof msg, &ctx->launches)
                     : rzw_optimize_each(dfft, obs->numbins, obs->lobin, cands + c0, c1 - c0, out + c0,
                                         ctx->tw_rzw.p, budget, ctx->stream, msg, sizeof msg,
                                         &ctx->launches);
            if (rc) return fail(ctx, rc, "%s", msg);
            c0 = c1;
        }
        return AB_OK;
    }
    // -noharmpolish (src/accel_utils.c:585-611): max_rz_arr for each harmonic
    // on its own at (r h, z h); results gathered back per candidate below
    const bool each = obs->noharmpolish != 0;
    std::vector<PolishIn> in;
    std::vector<long long> owner;
    for (long long k = 0; k < n; k++) {
        if (!each) {
            in.push_back(PolishIn{cands[k].r, cands[k].z, cands[k].numharm, 0});
            continue;
        }
        for (int ii = 0; ii < cands[k].numharm; ii++) {
            in.push_back(PolishIn{cands[k].r * (ii + 1), cands[k].z * (ii + 1), 1, 1});
            owner.push_back(k);
        }
    }
    const long long nin = (long long) in.size();
    if (nin > (1 << 24)) return fail(ctx, AB_ERR_ARG, "too many harmonics to polish");
    std::vector<ab_polished> single(each ? (size_t) nin : 0);
    ab_polished *hout = each ? single.data() : out;
    DevBuf<PolishIn> din;
    DevBuf<ab_polished> dout;
    cudaError_t e = din.ensure((size_t) nin);
    if (e == cudaSuccess) e = dout.ensure((size_t) nin);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(din.p, in.data(), sizeof(PolishIn) * nin, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
        e = launch_polish(dfft, obs->numbins, obs->lobin, din.p, (int) nin, dout.p, ctx->stream);
    if (e == cudaSuccess) ctx->launches++;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(hout, dout.p, sizeof(ab_polished) * nin, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    din.release();
    dout.release();
    if (e != cudaSuccess) return fail(ctx, AB_ERR_CUDA, "candidate polishing failed: %s", cudaGetErrorString(e));
    if (each) {
        for (long long k = 0; k < n; k++) {
            memset(&out[k], 0, sizeof out[k]);
            out[k].numharm = cands[k].numharm;
        }
        std::vector<int> seen((size_t) n, 0);
        for (long long q = 0; q < nin; q++) {
            const long long k = owner[q];
            const int ii = seen[k]++;
            out[k].pows[ii] = single[q].pows[0];
            out[k].hirs[ii] = single[q].hirs[0];      // r + lobin of the harmonic's own optimum
            out[k].hizs[ii] = single[q].hizs[0];
            out[k].hiws[ii] = 0.0;
            out[k].derivs[ii] = single[q].derivs[0];
        }
    }
    return AB_OK;
}

// ---- time-series input path ------------------------------------------------
static int realfft_dev(ab_ctx *ctx, const float *series, long long n, int series_on_device, float2 *dout)
{
    if (!realfft_supported(n))
        return fail(ctx, AB_ERR_ARG, "realfft length %lld: need an even length from 1024 to 2^26 "
                                     "(n/2 a power of two up to 2^26, else up to 2^25)", n);
    const float *din = series;
    if (!series_on_device || misaligned8(series)) {
        // host series, or a device series not on an 8-byte boundary (the
        // transforms read it in pairs): into the aligned input buffer
        CK(ctx->ser_in.ensure((size_t) ((n + 1) / 2)));
        CK(cudaMemcpyAsync(ctx->ser_in.p, series, sizeof(float) * n,
                           series_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                           ctx->stream));
        din = reinterpret_cast<const float *>(ctx->ser_in.p);
    }
    const long long M = n / 2;
    if (pow2_fft_supported(M)) {
        CK(ctx->ser_scr.ensure((size_t) M));
        CK(launch_realfft(din, dout, ctx->ser_scr.p, n, ctx->stream));
        ctx->launches += 6;
        return AB_OK;
    }
    const long long L = bluestein_len(M);
    CK(ctx->ser_scr.ensure((size_t) L));
    CK(ctx->blu_a.ensure((size_t) L));
    const bool fresh = ctx->blu_M != M || ctx->blu_b.n < (size_t) L;
    CK(ctx->blu_b.ensure((size_t) L));
    CK(launch_realfft_bluestein(din, dout, ctx->blu_a.p, ctx->ser_scr.p, ctx->blu_b.p, fresh, n,
                                ctx->stream));
    ctx->blu_M = M;
    ctx->launches += fresh ? 24 : 17;
    return AB_OK;
}

static int deredden_dev(ab_ctx *ctx, float2 *dfft, long long numbins, int startwidth, int endwidth,
                        double endfreq, double T)
{
    if (endwidth > AB_DERED_MAXW)
        return fail(ctx, AB_ERR_ARG, "deredden endwidth %d above %d", endwidth, AB_DERED_MAXW);
    long long nb = 0;
    int rc = ab_dered_plan(numbins, startwidth, endwidth, endfreq, T, nullptr, 0, &nb);
    if (rc) return fail(ctx, rc, "deredden: spectrum of %lld bins too short", numbins);
    if (nb > (1LL << 30)) return fail(ctx, AB_ERR_ARG, "deredden: too many blocks");
    std::vector<int> plan((size_t) (2 * nb));
    ab_dered_plan(numbins, startwidth, endwidth, endfreq, T, plan.data(), nb, &nb);
    CK(ctx->dered_blocks.ensure((size_t) nb));
    CK(ctx->dered_means.ensure((size_t) nb));
    CK(cudaMemcpyAsync(ctx->dered_blocks.p, plan.data(), sizeof(int) * 2 * nb, cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(launch_deredden(dfft, ctx->dered_blocks.p, (int) nb, ctx->dered_means.p, ctx->stream));
    ctx->launches += 2;
    // the plan upload is pageable: wait before the vector goes away
    CK(cudaStreamSynchronize(ctx->stream));
    return AB_OK;
}

int ab_realfft(ab_ctx *ctx, const float *series, long long n, int series_on_device, ab_fcomplex *out,
               int out_on_device)
{
    if (!ctx || !series || !out) return AB_ERR_ARG;
    int rc = use_device(ctx);
    if (rc) return rc;
    float2 *dout = reinterpret_cast<float2 *>(out);
    if (!out_on_device) {
        CK(ctx->fft.ensure((size_t) (n / 2)));
        dout = ctx->fft.p;
        ctx->fft_valid = false;
    }
    rc = realfft_dev(ctx, series, n, series_on_device, dout);
    if (rc) return rc;
    if (!out_on_device)
        CK(cudaMemcpyAsync(out, dout, sizeof(float2) * (n / 2), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return AB_OK;
}

int ab_deredden(ab_ctx *ctx, ab_fcomplex *fft, long long numbins, int startwidth, int endwidth,
                double endfreq, double T, int fft_on_device)
{
    if (!ctx || !fft || numbins < 1) return AB_ERR_ARG;
    if (fft_on_device && misaligned8(fft))
        return fail(ctx, AB_ERR_ARG, "device spectrum not 8-byte aligned");
    int rc = use_device(ctx);
    if (rc) return rc;
    float2 *d = reinterpret_cast<float2 *>(fft);
    if (!fft_on_device) {
        CK(ctx->fft.ensure((size_t) numbins));
        ctx->fft_valid = false;
        d = ctx->fft.p;
        CK(cudaMemcpyAsync(d, fft, sizeof(float2) * numbins, cudaMemcpyHostToDevice, ctx->stream));
    }
    rc = deredden_dev(ctx, d, numbins, startwidth, endwidth, endfreq, T);
    if (rc) return rc;
    if (!fft_on_device)
        CK(cudaMemcpyAsync(fft, d, sizeof(float2) * numbins, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return AB_OK;
}

int ab_series_to_fft(ab_ctx *ctx, const float *series, long long n, double dt, int series_on_device,
                     ab_fcomplex *out, int out_on_device)
{
    if (!ctx || !series || !out || dt <= 0.0) return AB_ERR_ARG;
    if (out_on_device && misaligned8(out))
        return fail(ctx, AB_ERR_ARG, "device spectrum not 8-byte aligned");
    int rc = use_device(ctx);
    if (rc) return rc;
    float2 *dout = reinterpret_cast<float2 *>(out);
    if (!out_on_device) {
        CK(ctx->fft.ensure((size_t) (n / 2)));
        dout = ctx->fft.p;
        ctx->fft_valid = false;
    }
    rc = realfft_dev(ctx, series, n, series_on_device, dout);
    if (rc) return rc;
    rc = deredden_dev(ctx, dout, n / 2, 6, 200, 0.5 / dt, dt * (double) n);
    if (rc) return rc;
    if (!out_on_device)
        CK(cudaMemcpyAsync(out, dout, sizeof(float2) * (n / 2), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return AB_OK;
}

int ab_dedisperse(ab_ctx *ctx, const float *data, int data_on_device, long long nspec, int nchan,
                  double lofreq, double chanwidth, double dt, int nsub, const double *dms, int ndm,
                  int downsamp, float *out, int out_on_device)
{
    if (!ctx || !data || !out || !dms || nspec < 1 || nchan < 1 || nsub < 1 || ndm < 1 ||
        downsamp < 1 || nchan % nsub || nsub > 1024)
        return fail(ctx, AB_ERR_ARG, "dedispersion arguments");
    int rc = use_device(ctx);
    if (rc) return rc;
    const long long nout = nspec / downsamp;
    if (nout < 1) return fail(ctx, AB_ERR_ARG, "fewer samples than the downsampling factor");
    std::vector<int> cd((size_t) nchan), off((size_t) ndm * nsub);
    rc = ab_dedisp_delays(nchan, lofreq, chanwidth, dt, nsub, dms, ndm, downsamp, cd.data(),
                          off.data());
    if (rc) return fail(ctx, rc, "dedispersion delays (channels ascending in frequency, "
                                 "delays below 2^30 samples)");
    const size_t nx = (size_t) nspec * nchan;
    CK(ctx->dd_cd.ensure(cd.size()));
    CK(ctx->dd_off.ensure(off.size()));
    CK(cudaMemcpyAsync(ctx->dd_cd.p, cd.data(), sizeof(int) * cd.size(), cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(cudaMemcpyAsync(ctx->dd_off.p, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice,
                       ctx->stream));
    const float *dx = data;
    if (!data_on_device) {
        CK(ctx->dd_x.ensure(nx));
        rc = h2d_staged(ctx, ctx->dd_x.p, data, sizeof(float) * nx);
        if (rc) return rc;
        dx = ctx->dd_x.p;
    }
    CK(ctx->dd_sub.ensure((size_t) nsub * (size_t) dedisp_sub_pitch(nout)));
    float *dout = out;
    if (!out_on_device) {
        CK(ctx->dd_out.ensure((size_t) ndm * nout));
        dout = ctx->dd_out.p;
    }
    const int maxcd = *std::max_element(cd.begin(), cd.end());
    tick(ctx, 7, true);
    const cudaError_t le = launch_dedisp(dx, nspec, nchan, ctx->dd_cd.p, maxcd, nsub, downsamp,
                                         ctx->dd_off.p, off.data(), ndm, ctx->dd_sub.p, dout,
                                         ctx->stream);
    tick(ctx, 7, false);
    if (le != cudaSuccess)
        return fail(ctx, AB_ERR_ARG, "dedispersion launch refused (%s): a subband's channel delays "
                    "or a group of 8 consecutive DMs' subband offsets spread too far "
                    "for the shared-memory tiles (200 KB)",
                    cudaGetErrorString(le));
    ctx->launches += 2;
    if (!out_on_device)
        CK(cudaMemcpyAsync(out, dout, sizeof(float) * (size_t) ndm * nout, cudaMemcpyDeviceToHost,
                           ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));           // cd and off are host vectors
    harvest(ctx);
    return AB_OK;
}

int ab_search_dedispersed(ab_ctx *ctx, const float *data, int data_on_device, long long nspec,
                          int nchan, double lofreq, double chanwidth, double dt, int nsub,
                          const double *dms, int ndm, int downsamp, const ab_obs *obs,
                          ab_cand *cands, long long maxcands, long long *first)
{
    if (!ctx || !data || !dms || !obs || !first || ndm < 1 || downsamp < 1 || nspec < 1)
        return fail(ctx, AB_ERR_ARG, "dedispersed-search arguments");
    const long long nout = nspec / downsamp;
    const long long n = nout & ~1LL;
    if (n < 2 || obs->N != n || obs->numbins > n / 2 ||
        std::fabs(obs->dt - dt * downsamp) > 1e-9 * dt * downsamp)
        return fail(ctx, AB_ERR_ARG, "obs must describe the trials: N = %lld, dt = %.9g", n,
                    dt * downsamp);
    int rc = use_device(ctx);
    if (rc) return rc;
    // the trials stay in the context's trial buffer, then one spectrum at a time
    CK(ctx->dd_out.ensure((size_t) ndm * (size_t) nout));
    rc = ab_dedisperse(ctx, data, data_on_device, nspec, nchan, lofreq, chanwidth, dt, nsub, dms,
                       ndm, downsamp, ctx->dd_out.p, 1);
    if (rc) return rc;
    CK(ctx->dd_fft.ensure((size_t) (n / 2)));
    std::vector<ab_cand> all;
    first[0] = 0;
    for (int d = 0; d < ndm; d++) {
        rc = ab_series_to_fft(ctx, ctx->dd_out.p + (size_t) d * (size_t) nout, n, dt * downsamp, 1,
                              reinterpret_cast<ab_fcomplex *>(ctx->dd_fft.p), 1);
        if (rc) return rc;
        long long nc = 0;
        rc = ab_search(ctx, obs, reinterpret_cast<const ab_fcomplex *>(ctx->dd_fft.p), 1, 0, -1,
                       nullptr, 0, &nc);
        if (rc) return rc;
        all.insert(all.end(), ctx->last_cands.begin(), ctx->last_cands.end());
        first[d + 1] = (long long) all.size();
    }
    const long long total = (long long) all.size();
    if (cands)
        for (long long i = 0; i < total && i < maxcands; i++) cands[i] = all[(size_t) i];
    if (cands && total > maxcands)
        return fail(ctx, AB_ERR_OVERFLOW, "%lld candidates > maxcands", total);
    return AB_OK;
}

int ab_zapbirds(ab_ctx *ctx, ab_fcomplex *fft, int fft_on_device, long long numbins, long long N,
                const double *lobins, const double *hibins, int numbirds, int *numzapped)
{
    if (!ctx || !fft || numbins < 0 || numbirds < 0 || (numbirds > 0 && (!lobins || !hibins)))
        return AB_ERR_ARG;
    if (!fft_on_device)
        return ab_zapbirds_host(fft, numbins, N, lobins, hibins, numbirds, numzapped);
    if (misaligned8(fft)) return fail(ctx, AB_ERR_ARG, "device spectrum not 8-byte aligned");
    int rc = use_device(ctx);
    if (rc) return rc;
    long long lo = 0, hi = 0;
    if (ab_zap_bounds(numbins, N, lobins, hibins, numbirds, &lo, &hi))
        return fail(ctx, AB_ERR_ARG, "a birdie lies outside the spectrum");
    if (numzapped) *numzapped = 0;
    if (hi <= lo) return AB_OK;
    // the bins the zapping reads (measurement windows) and writes, to the host
    std::vector<ab_fcomplex> span((size_t) (hi - lo));
    CK(cudaMemcpyAsync(span.data(), fft + lo, sizeof(ab_fcomplex) * span.size(),
                       cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    rc = ab_zapbirds_span(span.data(), lo, numbins, N, lobins, hibins, numbirds, numzapped);
    if (rc) return fail(ctx, rc, "zapping");
    // and the zapped bins back
    const double top = (double) (N / 2);
    for (int i = 0; i < numbirds; i++) {
        if (lobins[i] >= top) break;
        const double hb = hibins[i] >= top ? top - 1 : hibins[i];
        const long long a = (long long) floor(lobins[i]), b = (long long) ceil(hb);
        if (b - a < 1) continue;
        CK(cudaMemcpyAsync(fft + a, span.data() + (a - lo), sizeof(ab_fcomplex) * (size_t) (b - a),
                           cudaMemcpyHostToDevice, ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return AB_OK;
}

int ab_ctx_set_corr_path(ab_ctx *ctx, int path)
{
    if (!ctx || (path != AB_CORR_FFT && path != AB_CORR_TC_SPLIT_BF16 &&
                 path != AB_CORR_TC_SPLIT_FP16))
        return AB_ERR_ARG;
    ctx->corr_path = path;
    return AB_OK;
}

int ab_ctx_set_hbm_budget(ab_ctx *ctx, size_t bytes)
{
    if (!ctx || bytes == 0) return AB_ERR_ARG;
    ctx->hbm_budget = bytes;
    ctx->scratch_budget = std::min<size_t>(8ull << 30, bytes / 4);
    return AB_OK;
}

int ab_prepare(ab_ctx *ctx, const ab_obs *obs)
{
    if (!ctx || !obs) return AB_ERR_ARG;
    int rc = use_device(ctx);
    if (rc) return rc;
    rc = ensure_banks(ctx, obs);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    harvest(ctx);
    return AB_OK;
}

static int upload_spectrum(ab_ctx *ctx, const ab_obs *obs, const ab_fcomplex *fft)
{
    CK(ctx->fft.ensure((size_t) obs->numbins));
    CK(cudaMemcpyAsync(ctx->fft.p, fft, sizeof(float2) * obs->numbins, cudaMemcpyHostToDevice,
                       ctx->stream));
    ctx->fft_bins = obs->numbins;
    ctx->fft_valid = true;
    return AB_OK;
}

int ab_search(ab_ctx *ctx, const ab_obs *obs, const ab_fcomplex *fft, int fft_on_device,
              long long first_block, long long max_blocks, ab_cand *cands, long long maxcands,
              long long *numcands)
{
    if (!ctx || !obs || !fft) return fail(ctx, AB_ERR_ARG, "null argument");
    if (fft_on_device && misaligned8(fft))
        return fail(ctx, AB_ERR_ARG, "device spectrum not 8-byte aligned");
    const double t_start = now_ms();
    int rc = use_device(ctx);
    if (rc) return rc;
    rc = ensure_banks(ctx, obs);
    if (rc) return rc;
    const float2 *dfft;
    if (fft_on_device) {
        dfft = reinterpret_cast<const float2 *>(fft);
    } else {
        rc = upload_spectrum(ctx, obs, fft);
        if (rc) return rc;
        dfft = ctx->fft.p;
    }
    double replay_ms = 0.0;
    ab_list *l = nullptr;
    for (int attempt = 0;; attempt++) {
        l = ab_list_new();
        if (!l) return fail(ctx, AB_ERR_NOMEM, "candidate list");
        if (ctx->worklog_on) ab_list_worklog(l, 1, obs->T);
        ctx->overflow_need = 0;
        rc = search_core(ctx, obs, dfft, first_block, max_blocks, -1, l, &replay_ms);
        if (!rc) rc = check_device_error(ctx);
        if (rc == AB_ERR_OVERFLOW && ctx->overflow_need > ctx->hit_cap && attempt < 3) {
            // a batch crossed the threshold more often than the hit buffer
            // holds: grow it and search again
            CK(cudaStreamSynchronize(ctx->stream));
            unsigned want = ctx->hit_cap;
            while (want < ctx->overflow_need + ctx->overflow_need / 4) want *= 2;
            ctx->hit_cap = want;
            ab_list_free(l);
            continue;
        }
        break;
    }
    const double t_done = now_ms();
    harvest(ctx);
    if (ctx->prof) {
        ctx->kms[4] += t_done - t_start - replay_ms;   // host wall time outside the replay
        ctx->kms[5] += replay_ms;                      // sort + replay (overlaps the device)
        ctx->kn[4]++; ctx->kn[5]++;
    }
    if (rc) {
        ab_list_free(l);
        return rc;
    }
    long long n = ab_list_get(l, nullptr, 0);
    ctx->last_cands.resize((size_t) n);
    ab_list_get(l, ctx->last_cands.data(), n);
    {
        size_t wlen = 0;
        const char *wtext = ab_list_worklog_text(l, &wlen);
        ctx->last_worklog.assign(wtext, wlen);
    }
    ab_list_free(l);
    if (cands)
        for (long long i = 0; i < n && i < maxcands; i++) cands[i] = ctx->last_cands[i];
    if (numcands) *numcands = n;
    if (cands && n > maxcands) return fail(ctx, AB_ERR_OVERFLOW, "%lld candidates > maxcands", n);
    return AB_OK;
}

int ab_last_cands(ab_ctx *ctx, ab_cand *out, long long maxout, long long *numcands)
{
    if (!ctx) return AB_ERR_ARG;
    long long n = (long long) ctx->last_cands.size();
    if (out)
        for (long long i = 0; i < n && i < maxout; i++) out[i] = ctx->last_cands[i];
    if (numcands) *numcands = n;
    return (out && n > maxout) ? AB_ERR_OVERFLOW : AB_OK;
}

int ab_last_hits(ab_ctx *ctx, long long *block, int *stage, int *wi, int *zi, int *ri, float *power,
                 long long maxhits, long long *numhits)
{
    if (!ctx) return AB_ERR_ARG;
    if (ctx->hits_truncated)
        return fail(ctx, AB_ERR_STATE, "the last search kept only its latest batches of hits");
    long long n = (long long) ctx->hkeys.size();
    std::vector<size_t> order(n);
    for (long long i = 0; i < n; i++) order[i] = i;
    std::sort(order.begin(), order.end(),
              [&](size_t a, size_t b) { return ctx->hkeys[a] < ctx->hkeys[b]; });
    for (long long i = 0; i < n && i < maxhits; i++) {
        unsigned long long k = ctx->hkeys[order[i]];
        if (ri) ri[i] = (int) (k & 0xFFFF);
        k >>= AB_KEY_RBITS;
        if (zi) zi[i] = (int) (k & 0xFFF);
        k >>= AB_KEY_ZBITS;
        if (wi) wi[i] = (int) (k & 0x7F);
        k >>= AB_KEY_WBITS;
        if (stage) stage[i] = (int) (k & 0x7);
        k >>= AB_KEY_SBITS;
        if (block) block[i] = (long long) k;
        if (power) power[i] = ctx->hpows[order[i]];
    }
    if (numhits) *numhits = n;
    return n > maxhits ? AB_ERR_OVERFLOW : AB_OK;
}

int ab_block_stage_sums(ab_ctx *ctx, const ab_obs *obs, const ab_fcomplex *fft_host,
                        long long block, float *out, size_t capacity)
{
    if (!ctx || !obs || !fft_host || !out) return AB_ERR_ARG;
    int rc = use_device(ctx);
    if (rc) return rc;
    rc = ensure_banks(ctx, obs);
    if (rc) return rc;
    size_t need = (size_t) obs->numharmstages * (obs->numw > 0 ? obs->numw : 1) * obs->numz *
                  obs->corr_uselen;
    if (capacity < need) return fail(ctx, AB_ERR_OVERFLOW, "need %zu floats", need);
    rc = upload_spectrum(ctx, obs, fft_host);
    if (rc) return rc;
    rc = search_core(ctx, obs, ctx->fft.p, block, 1, block, nullptr);
    if (!rc) rc = check_device_error(ctx);
    if (rc) return rc;
    CK(cudaMemcpyAsync(out, ctx->dbg.p, sizeof(float) * need, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    harvest(ctx);
    return AB_OK;
}

int ab_set_spectrum(ab_ctx *ctx, const ab_obs *obs, const ab_fcomplex *fft_host)
{
    if (!ctx || !obs || !fft_host) return AB_ERR_ARG;
    int rc = use_device(ctx);
    if (rc) return rc;
    rc = upload_spectrum(ctx, obs, fft_host);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return AB_OK;
}

static int find_bank(const ab_bankset &bs, int numharm, int harmnum)
{
    for (int i = 0; i < bs.nbanks; i++)
        if (bs.b[i].numharm == numharm && bs.b[i].harmnum == harmnum) return i;
    return -1;
}

int ab_subharm_fderivs_vol(ab_ctx *ctx, const ab_obs *obs, int numharm, int harmnum,
                           double fullrlo, double fullrhi, ab_ffdotpows *out)
{
    if (!ctx || !obs || !out) return AB_ERR_ARG;
    if (!ctx->fft_valid || ctx->fft_bins != obs->numbins)
        return fail(ctx, AB_ERR_STATE, "no spectrum uploaded (ab_set_spectrum)");
    if (fullrhi != fullrlo + obs->rstep - AB_DR)
        return fail(ctx, AB_ERR_ARG, "fullrhi must be fullrlo + rstep - 0.5");
    int rc = use_device(ctx);
    if (rc) return rc;
    rc = ensure_banks(ctx, obs);
    if (rc) return rc;
    int k = find_bank(ctx->bs, numharm, harmnum);
    if (k < 0) return fail(ctx, AB_ERR_ARG, "no template bank for harmonic %d/%d", harmnum, numharm);
    const ab_bank &b = ctx->bs.b[k];
    ab_hgeom g = ab_harm_geom(fullrlo, fullrhi, numharm, harmnum, obs->zlo, obs->wlo,
                              obs->corr_uselen);
    size_t need = (size_t) b.nw * b.nz * g.numrs;
    if (g.numrs > b.numrs_max)
        return fail(ctx, AB_ERR_ARG, "block start %.1f is not on the search's block grid", fullrlo);
    out->rlo = g.rlo;
    out->zlo = g.zlo;
    out->wlo = g.wlo;
    out->numrs = g.numrs;
    out->numzs = b.nz;
    out->numws = b.nw;
    if (!out->powers || out->capacity < need)
        return fail(ctx, AB_ERR_OVERFLOW, "plane needs %zu floats", need);
    SearchConsts sc = make_consts(obs, ctx->bs);
    sc.inmem = 0;                              // the block plane, not the full plane
    CK(ctx->errw.ensure(1));
    CK(cudaMemsetAsync(ctx->errw.p, 0, sizeof(unsigned), ctx->stream));
    sc.err = ctx->errw.p;
    CK(ctx->startr.ensure(1));
    CK(cudaMemcpyAsync(ctx->startr.p, &fullrlo, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(ctx->planes.ensure((size_t) ctx->bs.plane_per_block));
    BlockBatch bb{ctx->startr.p, 0, 1, 0};
    if (ctx->corr_path != AB_CORR_FFT) {
        rc = ensure_tc(ctx);
        if (rc) return rc;
        CK(ctx->dtime.ensure((size_t) ctx->bs.dtime_per_block));
        std::vector<TcItem> tplan;
        build_tc_plan(ctx->cur_bank->tc, ctx->bs, 1, k, k + 1, tplan);
        CK(ctx->titems.ensure(tplan.size()));
        CK(cudaMemcpyAsync(ctx->titems.p, tplan.data(), sizeof(TcItem) * tplan.size(),
                           cudaMemcpyHostToDevice, ctx->stream));
        rc = run_tc(ctx, sc, bb, ctx->fft.p, k, k + 1, ctx->titems.p, (int) tplan.size(), ctx->planes.p,
                    ctx->bs.plane_per_block, nullptr);
        if (rc) return rc;
    } else {
        CK(ctx->xhat.ensure((size_t) ctx->bs.xhat_per_block));
        rc = run_prep(ctx, sc, bb, ctx->fft.p, k, k + 1);
        if (rc) return rc;
        CorrPlan plan;
        build_corr_plan(ctx->bs, sc, 1, k, k + 1, plan);
        CK(ctx->items.ensure(plan.items.size()));
        CK(cudaMemcpyAsync(ctx->items.p, plan.items.data(), sizeof(CorrItem) * plan.items.size(),
                           cudaMemcpyHostToDevice, ctx->stream));
        rc = run_corr(ctx, sc, bb, plan, ctx->items.p, ctx->planes.p, ctx->bs.plane_per_block, nullptr);
        if (rc) return rc;
    }
    CK(cudaMemcpy2DAsync(out->powers, sizeof(float) * g.numrs, ctx->planes.p + b.plane_off,
                         sizeof(float) * b.numrs_max, sizeof(float) * g.numrs, (size_t) b.nw * b.nz,
                         cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    harvest(ctx);
    return check_device_error(ctx);
}

int ab_add_ffdotpows(ab_ctx *ctx, const ab_obs *obs, ab_ffdotpows *fund, const ab_ffdotpows *sub,
                     int numharm, int harmnum, double fullrlo)
{
    if (!ctx || !obs || !fund || !sub) return AB_ERR_ARG;
    int rc = use_device(ctx);
    if (rc) return rc;
    size_t nf = (size_t) fund->numws * fund->numzs * fund->numrs;
    size_t ns = (size_t) sub->numws * sub->numzs * sub->numrs;
    CK(ctx->tmpa.ensure(nf));
    CK(ctx->tmpb.ensure(ns));
    CK(cudaMemcpyAsync(ctx->tmpa.p, fund->powers, nf * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->tmpb.p, sub->powers, ns * 4, cudaMemcpyHostToDevice, ctx->stream));
    double f = (double) harmnum / (double) numharm;
    CK(launch_add_ffdot(ctx->tmpa.p, ctx->tmpb.p, fund->numws, fund->numzs, fund->numrs, sub->numzs,
                        sub->numrs, f, fund->wlo, sub->wlo, fullrlo, sub->rlo, obs->zlo, sub->zlo,
                        ctx->stream));
    ctx->launches++;
    CK(cudaMemcpyAsync(fund->powers, ctx->tmpa.p, nf * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return AB_OK;
}

int ab_fund_to_ffdotplane(ab_ctx *ctx, const ab_obs *obs, const ab_ffdotpows *fund)
{
    if (!ctx || !obs || !fund || !obs->inmem) return AB_ERR_ARG;
    int rc = use_device(ctx);
    if (rc) return rc;
    long long rlen = (obs->highestbin + obs->corr_uselen) * (long long) AB_RDR;
    size_t rows = (size_t) obs->numz * rlen;
    bool fresh = ctx->fullplane.n < rows;
    CK(ctx->fullplane.ensure(rows));
    if (fresh) CK(cudaMemsetAsync(ctx->fullplane.p, 0, rows * sizeof(float), ctx->stream));
    if (fund->rlo * AB_RDR + fund->numrs > rlen) return fail(ctx, AB_ERR_ARG, "block beyond plane");
    CK(cudaMemcpy2DAsync(ctx->fullplane.p + fund->rlo * AB_RDR, sizeof(float) * rlen, fund->powers,
                         sizeof(float) * fund->numrs, sizeof(float) * fund->numrs, fund->numzs,
                         cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return AB_OK;
}

int ab_add_ffdotpows_ptrs(ab_ctx *ctx, const ab_obs *obs, ab_ffdotpows *fund,
                          const ab_ffdotpows *sub, int numharm, int harmnum, double fullrlo)
{
    return ab_add_ffdotpows(ctx, obs, fund, sub, numharm, harmnum, fullrlo);
}

int ab_fund_to_ffdotplane_trans(ab_ctx *ctx, const ab_obs *obs, const ab_ffdotpows *fund)
{
    return ab_fund_to_ffdotplane(ctx, obs, fund);
}

int ab_inmem_add_ffdotpows_trans(ab_ctx *ctx, const ab_obs *obs, ab_ffdotpows *fund, int numharm,
                                 int harmnum)
{
    return ab_inmem_add_ffdotpows(ctx, obs, fund, numharm, harmnum);
}

int ab_inmem_add_ffdotpows(ab_ctx *ctx, const ab_obs *obs, ab_ffdotpows *fund, int numharm,
                           int harmnum)
{
    if (!ctx || !obs || !fund || !obs->inmem) return AB_ERR_ARG;
    int rc = use_device(ctx);
    if (rc) return rc;
    long long rlen = (obs->highestbin + obs->corr_uselen) * (long long) AB_RDR;
    if (ctx->fullplane.n < (size_t) obs->numz * rlen)
        return fail(ctx, AB_ERR_STATE, "no in-memory plane (ab_fund_to_ffdotplane)");
    size_t nf = (size_t) fund->numzs * fund->numrs;
    CK(ctx->tmpa.ensure(nf));
    CK(cudaMemcpyAsync(ctx->tmpa.p, fund->powers, nf * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(launch_inmem_add(ctx->tmpa.p, ctx->fullplane.p, rlen, fund->numzs, fund->numrs,
                        (int) fund->rlo, fund->zlo, (double) harmnum / (double) numharm, ctx->stream));
    ctx->launches++;
    CK(cudaMemcpyAsync(fund->powers, ctx->tmpa.p, nf * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return AB_OK;
}

ab_candlist *ab_candlist_new(void) { return ab_list_new(); }
void ab_candlist_free(ab_candlist *l) { ab_list_free(l); }
long long ab_candlist_get(const ab_candlist *l, ab_cand *out, long long maxout)
{
    return ab_list_get(l, out, maxout);
}

int ab_candlist_insert(ab_candlist *l, float power, float sigma, int numharm, double r, double z,
                       double w)
{
    if (!l) return AB_ERR_ARG;
    return ab_list_insert(l, power, sigma, numharm, r, z, w);
}

// Threshold crossings of one host plane in the reference's visit order
// (w, z, r: src/accel_utils.c:1418-1433) with their candidate coordinates
// and sigma; the plane is copied to the device, thresholded there and the
// crossings come back.
static int plane_hits(ab_ctx *ctx, const ab_obs *obs, const ab_ffdotpows *ffd, int numharm,
                      std::vector<ab_cand> &out)
{
    out.clear();
    int rc = use_device(ctx);
    if (rc) return rc;
    int stage = 0;
    while ((1 << stage) < numharm) stage++;
    if ((1 << stage) != numharm || stage >= obs->numharmstages) return fail(ctx, AB_ERR_ARG, "numharm");
    size_t n = (size_t) ffd->numws * ffd->numzs * ffd->numrs;
    CK(ctx->tmpa.ensure(n));
    CK(cudaMemcpyAsync(ctx->tmpa.p, ffd->powers, n * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(ctx->keys.ensure(ctx->hit_cap));
    CK(ctx->pows.ensure(ctx->hit_cap));
    CK(ctx->count.ensure(1));
    CK(cudaMemsetAsync(ctx->count.p, 0, sizeof(unsigned), ctx->stream));
    HitBuf hb{ctx->keys.p, ctx->pows.p, ctx->count.p, ctx->hit_cap};
    CK(launch_threshold(ctx->tmpa.p, ffd->numws, ffd->numzs, ffd->numrs, obs->powcut[stage], stage,
                        hb, ctx->stream));
    ctx->launches++;
    long long nh = 0;
    rc = fetch_hits(ctx, &nh);
    if (rc) return rc;
    // keys hold (stage, w, z, r) with block 0; the plane's own rlo/zlo/wlo
    // give the candidate coordinates (src/accel_utils.c:1431-1433)
    std::vector<size_t> order(nh);
    for (long long i = 0; i < nh; i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return ctx->hkeys[a] < ctx->hkeys[b]; });
    for (long long i = 0; i < nh; i++) {
        unsigned long long k = ctx->hkeys[order[i]];
        int ri = (int) (k & 0xFFFF);
        k >>= AB_KEY_RBITS;
        int zi = (int) (k & 0xFFF);
        k >>= AB_KEY_ZBITS;
        int wi = (int) (k & 0x7F);
        float pw = ctx->hpows[order[i]];
        float sig = (float) ab_candidate_sigma(pw, numharm, (double) obs->numindep[stage]);
        double rr = (ffd->rlo + ri * (double) AB_DR) / (double) numharm;
        double zz = (ffd->zlo + zi * (double) AB_DZ) / (double) numharm;
        double ww = (ffd->wlo + wi * (double) AB_DW) / (double) numharm;
        out.push_back(ab_cand{pw, sig, numharm, rr, zz, ww});
    }
    return AB_OK;
}

int ab_search_ffdotpows(ab_ctx *ctx, const ab_obs *obs, const ab_ffdotpows *ffd, int numharm,
                        ab_candlist *list)
{
    if (!ctx || !obs || !ffd || !list) return AB_ERR_ARG;
    std::vector<ab_cand> hits;
    int rc = plane_hits(ctx, obs, ffd, numharm, hits);
    if (rc) return rc;
    for (const ab_cand &h : hits)
        if (ab_list_insert(list, h.power, h.sigma, numharm, h.r, h.z, h.w) < 0)
            return fail(ctx, AB_ERR_NOMEM, "candidate list");
    return AB_OK;
}

int ab_ffdot_hits(ab_ctx *ctx, const ab_obs *obs, const ab_ffdotpows *ffd, int numharm,
                  ab_cand *out, long long maxout, long long *numhits)
{
    if (!ctx || !obs || !ffd || !numhits || (maxout > 0 && !out)) return AB_ERR_ARG;
    std::vector<ab_cand> hits;
    int rc = plane_hits(ctx, obs, ffd, numharm, hits);
    *numhits = (long long) hits.size();
    if (rc) return rc;
    for (long long i = 0; i < (long long) hits.size() && i < maxout; i++) out[i] = hits[i];
    return (long long) hits.size() > maxout ? AB_ERR_OVERFLOW : AB_OK;
}

int ab_set_worklog(ab_ctx *ctx, int on)
{
    if (!ctx) return AB_ERR_ARG;
    ctx->worklog_on = on ? 1 : 0;
    return AB_OK;
}

int ab_last_worklog(ab_ctx *ctx, char *out, size_t cap, size_t *len)
{
    if (!ctx || !len) return AB_ERR_ARG;
    *len = ctx->last_worklog.size();
    if (out && cap) {
        const size_t k = std::min(cap - 1, ctx->last_worklog.size());
        memcpy(out, ctx->last_worklog.data(), k);
        out[k] = '\0';
    }
    return AB_OK;
}

int ab_candlist_set_worklog(ab_candlist *l, int on, double T)
{
    if (!l || (on && !(T > 0.0))) return AB_ERR_ARG;
    ab_list_worklog(l, on, T);
    return AB_OK;
}

long long ab_candlist_worklog(const ab_candlist *l, char *out, size_t cap)
{
    if (!l) return AB_ERR_ARG;
    size_t len = 0;
    const char *t = ab_list_worklog_text(l, &len);
    if (out && cap) {
        const size_t k = len < cap - 1 ? len : cap - 1;
        memcpy(out, t, k);
        out[k] = '\0';
    }
    return (long long) len;
}

int ab_gen_response(ab_ctx *ctx, double roffset, int numbetween, double z, double w, int numkern,
                    ab_fcomplex *out)
{
    if (!ctx || !out) return AB_ERR_ARG;
    if (roffset < 0.0 || roffset >= 1.0 || numbetween < 1 || numbetween >= 20000 ||
        numkern < numbetween || numkern % (2 * numbetween))
        return fail(ctx, AB_ERR_ARG, "bad response arguments (src/responses.c:344-360)");
    int rc = use_device(ctx);
    if (rc) return rc;
    if ((rc = ensure_tw64(ctx))) return rc;
    CK(ctx->resp.ensure((size_t) numkern));
    cudaError_t e = launch_response(roffset, numbetween, z, w, numkern, ctx->resp.p, ctx->tw64.p,
                                    kTwLog2, nullptr, ctx->stream);
    if (e != cudaSuccess) return fail(ctx, AB_ERR_ARG, "response generation: %s", cudaGetErrorString(e));
    ctx->launches++;
    CK(cudaMemcpyAsync(out, ctx->resp.p, sizeof(float2) * numkern, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return AB_OK;
}

int ab_bank_kernel(ab_ctx *ctx, const ab_obs *obs, int numharm, int harmnum, int wi, int zi,
                   ab_fcomplex *out, int maxlen, int *fftlen_dev)
{
    if (!ctx || !obs) return AB_ERR_ARG;
    int rc = use_device(ctx);
    if (rc) return rc;
    rc = ensure_banks(ctx, obs);
    if (rc) return rc;
    int k = find_bank(ctx->bs, numharm, harmnum);
    if (k < 0) return fail(ctx, AB_ERR_ARG, "no bank %d/%d", harmnum, numharm);
    const ab_bank &b = ctx->bs.b[k];
    if (fftlen_dev) *fftlen_dev = b.L;
    if (wi < 0 || wi >= b.nw || zi < 0 || zi >= b.nz) return fail(ctx, AB_ERR_ARG, "template index");
    if (!out) return AB_OK;
    if (maxlen < b.L) return fail(ctx, AB_ERR_OVERFLOW, "need %d", b.L);
    CK(cudaMemcpyAsync(out, ctx->tmpl_p + b.tmpl_off + (long long) (wi * b.nz + zi) * b.L,
                       sizeof(float2) * b.L, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    harvest(ctx);
    return AB_OK;
}

int ab_ctx_set_profiling(ab_ctx *ctx, int on)
{
    if (!ctx) return AB_ERR_ARG;
    ctx->prof = on != 0;
    return AB_OK;
}

int ab_ctx_kernel_times(ab_ctx *ctx, double *ms, long long *launches, int nkinds)
{
    if (!ctx) return AB_ERR_ARG;
    for (int i = 0; i < nkinds && i < kNumKinds; i++) {
        if (ms) ms[i] = ctx->kms[i];
        if (launches) launches[i] = ctx->kn[i];
    }
    return AB_OK;
}

int ab_ctx_reset_kernel_times(ab_ctx *ctx)
{
    if (!ctx) return AB_ERR_ARG;
    for (int i = 0; i < kNumKinds; i++) {
        ctx->kms[i] = 0;
        ctx->kn[i] = 0;
    }
    ctx->launches = 0;
    return AB_OK;
}

long long ab_ctx_launch_count(ab_ctx *ctx) { return ctx ? ctx->launches : -1; }

int ab_tc_gemm(ab_ctx *ctx, const float *A, const float *B, float *C, int N, int K, int split)
{
    if (!ctx || !A || !B || !C) return AB_ERR_ARG;
    int rc = use_device(ctx);
    if (rc) return rc;
    DevBuf<float> a, b, c;
    CK(a.ensure((size_t) 128 * K));
    CK(b.ensure((size_t) N * K));
    CK(c.ensure((size_t) 128 * N));
    CK(ctx->errw.ensure(1));
    CK(cudaMemsetAsync(ctx->errw.p, 0, sizeof(unsigned), ctx->stream));
    CK(cudaMemcpyAsync(a.p, A, sizeof(float) * 128 * K, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(b.p, B, sizeof(float) * N * K, cudaMemcpyHostToDevice, ctx->stream));
    cudaError_t e = launch_tc_gemm(a.p, b.p, c.p, N, K, split, ctx->errw.p, ctx->stream);
    if (e != cudaSuccess) return fail(ctx, AB_ERR_ARG, "tc gemm: %s", cudaGetErrorString(e));
    CK(cudaMemcpyAsync(C, c.p, sizeof(float) * 128 * N, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    a.release();
    b.release();
    c.release();
    return check_device_error(ctx);
}

int ab_measure_fp32_peak(ab_ctx *ctx, double *tflops)
{
    if (!ctx || !tflops) return AB_ERR_ARG;
    int rc = use_device(ctx);
    if (rc) return rc;
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    CK(ctx->tmpa.ensure(1));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    const int iters = 1 << 14;
    double best = 0.0;
    for (int k = 0; k < 7; k++) {
        cudaEventRecord(e0, ctx->stream);
        cudaError_t e = launch_fma_peak(ctx->tmpa.p, iters, sms, ctx->stream);
        cudaEventRecord(e1, ctx->stream);
        if (e != cudaSuccess) return fail(ctx, AB_ERR_CUDA, "fma probe: %s", cudaGetErrorString(e));
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        double fl = 2.0 * 8.0 * iters * 256.0 * 8.0 * sms;
        if (k >= 2 && ms > 0) best = std::max(best, fl / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *tflops = best;
    return AB_OK;
}

}  // extern "C"
