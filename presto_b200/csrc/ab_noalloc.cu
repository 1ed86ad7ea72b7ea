// ab_noalloc.cu -- plane generation for one block and one harmonic that
// allocates no memory.
//
// For callers that cannot call cudaMalloc: real-time pipelines that reserve
// all device memory at start-up and forbid allocation in their processing
// loop, hosts whose device memory belongs to another allocator (a framework's
// caching pool), and stream-ordered code where an allocation would
// synchronise the device.  The caller passes every input and output as a
// device pointer; the engine's own intermediates (the block's data spectrum,
// the bank descriptor, the block start and the correlation work list) live
// in a file-scope static device array instead of context memory.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <mutex>

#include "ab_host.h"
#include "ab_index.h"
#include "ab_kernels.h"

using namespace ab;

namespace {

// Static scratch: 192 KiB, held by every GPU that loads the library until exit
// (work items and a data spectrum of up to 4096 points, for 8192-point banks).
constexpr size_t kScratchBytes = 192u << 10;
constexpr size_t kDescOff = 0;          // ab_bank
constexpr size_t kStartOff = 1024;      // double
constexpr size_t kItemsOff = 2048;      // CorrItem[kMaxItems]
constexpr int kMaxItems = 8192;
constexpr size_t kXhatOff = kItemsOff + sizeof(CorrItem) * kMaxItems;   // float2[L/2]

static_assert(sizeof(ab_bank) <= kStartOff - kDescOff, "descriptor slot");

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// The array's device address, looked up (cudaGetSymbolAddress) on the first
// call in each CUDA context and cached by the context's process-unique ID
// (cuCtxGetId), so that a context created later on the same device -- after
// a cudaDeviceReset, or a caller's own driver-API context -- gets its own
// lookup instead of a stale address.  The two driver functions come through
// the runtime's entry-point query; the library does not link libcuda.
typedef int (*ctx_get_current_fn)(void **ctx);
typedef int (*ctx_get_id_fn)(void *ctx, unsigned long long *id);
constexpr int kCacheSlots = 64;
std::mutex g_mu;
ctx_get_current_fn g_get_current = nullptr;
ctx_get_id_fn g_get_id = nullptr;
bool g_entry_points_tried = false;
unsigned long long g_ctx_id[kCacheSlots];
void *g_scratch_addr[kCacheSlots];
int g_next_slot = 0;

// the current context's ID (0 when the thread has no current context yet)
bool current_ctx_id(unsigned long long *id)
{
    *id = 0;
    void *c = nullptr;
    if (g_get_current(&c) != 0) return false;
    if (c && g_get_id(c, id) != 0) return false;
    return true;
}

cudaError_t scratch_address(unsigned char **out)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_entry_points_tried) {
        g_entry_points_tried = true;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", (void **) &g_get_current, 12000,
                                             cudaEnableDefault, &q1) != cudaSuccess ||
            q1 != cudaDriverEntryPointSuccess)
            g_get_current = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", (void **) &g_get_id, 12000,
                                             cudaEnableDefault, &q2) != cudaSuccess ||
            q2 != cudaDriverEntryPointSuccess)
            g_get_id = nullptr;
    }
    if (!g_get_current || !g_get_id) return cudaErrorNotSupported;
    unsigned long long id = 0;
    if (!current_ctx_id(&id)) return cudaErrorDeviceUninitialized;
    if (id)
        for (int i = 0; i < kCacheSlots; i++)
            if (g_ctx_id[i] == id) {
                *out = static_cast<unsigned char *>(g_scratch_addr[i]);
                return cudaSuccess;
            }
    // first call in this context: the lookup also makes the runtime's
    // context current when the thread had none
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    if (!current_ctx_id(&id) || !id) return cudaErrorDeviceUninitialized;
    const int slot = g_next_slot;
    g_next_slot = (g_next_slot + 1) % kCacheSlots;
    g_ctx_id[slot] = id;
    g_scratch_addr[slot] = p;
    *out = static_cast<unsigned char *>(p);
    return cudaSuccess;
}

__global__ void k_noalloc_setup(ab_bank desc, double startr, int ntmpl, int tile, int nitems,
                                ab_bank *d_desc, double *d_start, CorrItem *d_items)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        *d_desc = desc;
        *d_start = startr;
    }
    if (i < nitems) {
        int t0 = i * tile;
        d_items[i] = CorrItem{0, 0, t0, min(tile, ntmpl - t0)};
    }
}

}  // namespace

extern "C" int ab_fderivs_vol_noalloc(const ab_obs *obs, int numharm, int harmnum,
                                      double fullrlo, const ab_fcomplex *d_fft,
                                      const ab_fcomplex *d_templates, size_t templates_capacity,
                                      float *d_powers, size_t powers_capacity, void *stream,
                                      ab_ffdotpows *meta_out)
{
    if (!obs || !d_fft || !d_templates || !d_powers) return AB_ERR_ARG;
    // complex arrays are read as 8-byte pairs, powers as 4-byte words: a
    // pointer off those boundaries would fault the kernels
    if ((reinterpret_cast<uintptr_t>(d_fft) | reinterpret_cast<uintptr_t>(d_templates)) & 7u ||
        reinterpret_cast<uintptr_t>(d_powers) & 3u)
        return AB_ERR_ARG;
    // a CUDA error left pending by the caller's own work stays the caller's:
    // nothing is launched, so no error check below can consume it
    if (cudaPeekAtLastError() != cudaSuccess) return AB_ERR_STATE;
    ab_bankset bs;
    if (ab_bankset_init(obs, &bs) != AB_OK) return AB_ERR_ARG;
    int k = -1;
    for (int i = 0; i < bs.nbanks; i++)
        if (bs.b[i].numharm == numharm && bs.b[i].harmnum == harmnum) k = i;
    if (k < 0) return AB_ERR_ARG;
    ab_bank b = bs.b[k];
    const double fullrhi = fullrlo + obs->rstep - AB_DR;
    const ab_hgeom g = ab_harm_geom(fullrlo, fullrhi, numharm, harmnum, obs->zlo, obs->wlo,
                                    obs->corr_uselen);
    const size_t need = (size_t) b.nw * b.nz * g.numrs;
    if (meta_out) {
        meta_out->rlo = g.rlo;
        meta_out->zlo = g.zlo;
        meta_out->wlo = g.wlo;
        meta_out->numrs = g.numrs;
        meta_out->numzs = b.nz;
        meta_out->numws = b.nw;
    }
    if (g.numrs > b.numrs_max) return AB_ERR_ARG;
    const int G = b.L >= 4096 ? 1 : 4096 / b.L, tile = 16 * G;
    const int nitems = (b.ntmpl + tile - 1) / tile;
    if (nitems > kMaxItems || kXhatOff + sizeof(float2) * (size_t) (b.L / 2) > kScratchBytes) {
        fprintf(stderr, "ab_fderivs_vol_noalloc: bank %d/%d needs %d work items and a %d-point "
                        "spectrum; the static scratch holds %d items and %zu bytes\n",
                harmnum, numharm, nitems, b.L / 2, kMaxItems, kScratchBytes);
        return AB_ERR_BUDGET;
    }
    // the template length follows the process-wide transform-cost table: a
    // table changed since the caller built its templates changes L, which
    // the capacity check catches before anything reads past them
    if (templates_capacity < (size_t) b.ntmpl * b.L) return AB_ERR_ARG;
    if (powers_capacity < need) return AB_ERR_OVERFLOW;
    unsigned char *scr = nullptr;
    if (scratch_address(&scr) != cudaSuccess) return AB_ERR_CUDA;
    ab_bank *d_desc = reinterpret_cast<ab_bank *>(scr + kDescOff);
    double *d_start = reinterpret_cast<double *>(scr + kStartOff);
    CorrItem *d_items = reinterpret_cast<CorrItem *>(scr + kItemsOff);
    float2 *d_xhat = reinterpret_cast<float2 *>(scr + kXhatOff);

    // The caller's arrays: templates [nw][nz][L] at offset 0, powers
    // [nw][nz][numrs] (row stride numrs), data spectrum at scratch offset 0.
    b.tmpl_off = 0;
    b.plane_off = 0;
    b.xhat_off = 0;
    b.numrs_max = g.numrs;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_noalloc_setup<<<(nitems + 255) / 256, 256, 0, st>>>(b, fullrlo, b.ntmpl, tile, nitems,
                                                           d_desc, d_start, d_items);
    if (cudaGetLastError() != cudaSuccess) return AB_ERR_CUDA;

    SearchConsts sc{};
    sc.obs_zlo = obs->zlo;
    sc.obs_wlo = obs->wlo;
    sc.obs_rlo = obs->rlo;
    sc.obs_lobin = obs->lobin;
    sc.numbins = obs->numbins;
    sc.rlen = (obs->highestbin + obs->corr_uselen) * (long long) AB_RDR;
    sc.corr_uselen = obs->corr_uselen;
    sc.rstep = obs->rstep;
    sc.numz = obs->numz;
    sc.numws = obs->numw > 0 ? obs->numw : 1;
    sc.stages = obs->numharmstages;
    sc.inmem = 0;
    sc.nbanks = 1;
    sc.nph = obs->nph;
    sc.norm_type = obs->norm_type;
    BlockBatch bb{d_start, 0, 1, 0};
    if (launch_prep(d_desc, &b, 1, sc, bb, reinterpret_cast<const float2 *>(d_fft), d_xhat,
                    b.L / 2, nullptr, st) != cudaSuccess)
        return AB_ERR_CUDA;
    if (launch_corr(b.L, d_desc, sc, bb, d_items, nitems, d_xhat, b.L / 2,
                    reinterpret_cast<const float2 *>(d_templates), d_powers, 0, nullptr,
                    st) != cudaSuccess)
        return AB_ERR_CUDA;
    return AB_OK;
}
