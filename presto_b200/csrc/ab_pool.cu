// ab_pool.cu -- batched and served searches: a pool of worker threads, each
// owning an engine context (its own stream, template-bank cache and scratch)
// on one device.  Requests (one spectrum + accelsearch options each) queue in
// arrival order; a worker takes the head request as soon as it is free and the
// request's device-memory footprint fits the pool's HBM budget, so requests
// that arrive while others run are admitted as workers and memory free up and
// their kernels overlap on the GPU.  Each request's result is exactly the
// plain single-request search (the worker runs ab_search on it).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "ab_host.h"

namespace {

double wall_ms()
{
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

struct Request {
    long long id = 0;
    ab_obs obs{};
    std::vector<ab_fcomplex> fft;
    size_t plane_bytes = 0;     // in-memory f-fdot plane the search needs
    size_t input_bytes = 0;     // spectrum on the device
    double t_submit = 0, t_start = 0, t_done = 0;
    int rc = AB_OK;
    std::string err;
    std::vector<ab_cand> cands;
    bool done = false;
};

}  // namespace

struct ab_pool {
    int device = 0;
    size_t budget = 0;          // bytes the pool may hold on the device
    size_t reserved = 0;        // per-worker fixed parts (scratch, hits, templates)
    std::vector<ab_ctx *> ctxs;
    std::vector<size_t> held_plane;   // in-memory plane capacity each worker holds
    std::vector<std::thread> threads;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> queue;
    std::map<long long, Request *> reqs;
    size_t active_input = 0;
    long long next_id = 1;
    bool stop = false;
    std::string err;
    std::vector<double> latencies;
    double busy_first = -1, busy_last = 0;
    long long completed = 0;
};

static size_t plane_bytes(const ab_obs &o)
{
    if (!o.inmem) return 0;
    return sizeof(float) * (size_t) o.numz * (size_t) ((o.highestbin + o.corr_uselen) * 2);
}

// Memory the pool would hold if worker w took request r.
static size_t need_if(const ab_pool *p, int w, const Request *r)
{
    size_t held = 0;
    for (size_t x : p->held_plane) held += x;
    size_t grow = r->plane_bytes > p->held_plane[w] ? r->plane_bytes - p->held_plane[w] : 0;
    return p->reserved + held + grow + p->active_input + r->input_bytes;
}

static void worker_main(ab_pool *p, int w)
{
    ab_ctx *ctx = p->ctxs[w];
    for (;;) {
        Request *r = nullptr;
        {
            std::unique_lock<std::mutex> lk(p->mu);
            p->cv_work.wait(lk, [&] {
                return p->stop || (!p->queue.empty() && need_if(p, w, p->queue.front()) <= p->budget);
            });
            if (p->stop) return;
            r = p->queue.front();
            p->queue.pop_front();
            if (r->plane_bytes > p->held_plane[w]) p->held_plane[w] = r->plane_bytes;
            p->active_input += r->input_bytes;
            r->t_start = wall_ms();
            if (p->busy_first < 0) p->busy_first = r->t_start;
        }
        long long n = 0;
        int rc = ab_search(ctx, &r->obs, r->fft.data(), 0, 0, -1, nullptr, 0, &n);
        std::vector<ab_cand> out;
        if (rc == AB_OK) {
            out.resize((size_t) n);
            rc = ab_last_cands(ctx, out.data(), n, &n);
        }
        std::string msg = rc ? ab_ctx_last_error(ctx) : "";
        {
            std::lock_guard<std::mutex> lk(p->mu);
            r->rc = rc;
            r->err = msg;
            r->cands.swap(out);
            r->fft.clear();
            r->fft.shrink_to_fit();
            r->t_done = wall_ms();
            r->done = true;
            p->active_input -= r->input_bytes;
            p->latencies.push_back(r->t_done - r->t_submit);
            p->busy_last = r->t_done;
            p->completed++;
        }
        p->cv_done.notify_all();
        p->cv_work.notify_all();
    }
}

extern "C" {

int ab_pool_create(int device, int nworkers, size_t hbm_budget, ab_pool **out)
{
    if (!out || nworkers < 1 || nworkers > 64) return AB_ERR_ARG;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return AB_ERR_CUDA;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return AB_ERR_CUDA;
    ab_pool *p = new ab_pool();
    p->device = device;
    p->budget = hbm_budget ? hbm_budget : (size_t) (0.8 * (double) fr);
    // per worker: block scratch, two hit sets, template cache, spectrum slot
    size_t scratch = std::min<size_t>(8ull << 30, p->budget / (4 * (size_t) nworkers));
    size_t per_worker = scratch + (256ull << 20) + (1ull << 30);
    p->reserved = per_worker * (size_t) nworkers;
    if (p->reserved >= p->budget) {
        delete p;
        return AB_ERR_BUDGET;
    }
    for (int w = 0; w < nworkers; w++) {
        ab_ctx *c = nullptr;
        int rc = ab_ctx_create(device, &c);
        if (rc) {
            for (auto *x : p->ctxs) ab_ctx_destroy(x);
            delete p;
            return rc;
        }
        ab_ctx_set_hbm_budget(c, 4 * scratch);    // a context's scratch is budget / 4
        p->ctxs.push_back(c);
        p->held_plane.push_back(0);
    }
    for (int w = 0; w < nworkers; w++) p->threads.emplace_back(worker_main, p, w);
    *out = p;
    return AB_OK;
}

void ab_pool_destroy(ab_pool *p)
{
    if (!p) return;
    {
        std::lock_guard<std::mutex> lk(p->mu);
        p->stop = true;
    }
    p->cv_work.notify_all();
    for (auto &t : p->threads) t.join();
    for (auto *c : p->ctxs) ab_ctx_destroy(c);
    for (auto &kv : p->reqs) delete kv.second;
    for (auto *r : p->queue)
        if (!p->reqs.count(r->id)) delete r;
    delete p;
}

const char *ab_pool_last_error(const ab_pool *p) { return p ? p->err.c_str() : "no pool"; }

int ab_pool_set_corr_path(ab_pool *p, int path)
{
    if (!p) return AB_ERR_ARG;
    std::lock_guard<std::mutex> lk(p->mu);
    if (!p->queue.empty()) {
        p->err = "the correlation path is set before requests are submitted";
        return AB_ERR_STATE;
    }
    for (auto *c : p->ctxs) {
        int rc = ab_ctx_set_corr_path(c, path);
        if (rc) return rc;
    }
    return AB_OK;
}

int ab_pool_submit(ab_pool *p, const ab_params *params, const ab_fcomplex *fft, long long *ticket)
{
    if (!p || !params || !fft || !ticket) return AB_ERR_ARG;
    Request *r = new Request();
    int rc = ab_obs_init(params, &r->obs);
    if (rc) {
        delete r;
        std::lock_guard<std::mutex> lk(p->mu);
        p->err = "invalid search options";
        return rc;
    }
    r->plane_bytes = plane_bytes(r->obs);
    r->input_bytes = sizeof(ab_fcomplex) * (size_t) r->obs.numbins;
    {
        std::lock_guard<std::mutex> lk(p->mu);
        if (p->reserved + r->plane_bytes + r->input_bytes > p->budget) {
            p->err = "request needs more device memory than the pool's budget";
            delete r;
            return AB_ERR_BUDGET;
        }
    }
    r->fft.assign(fft, fft + r->obs.numbins);
    {
        std::lock_guard<std::mutex> lk(p->mu);
        r->id = p->next_id++;
        r->t_submit = wall_ms();
        p->reqs[r->id] = r;
        p->queue.push_back(r);
        *ticket = r->id;
    }
    p->cv_work.notify_all();
    return AB_OK;
}

int ab_pool_wait(ab_pool *p, long long ticket, ab_cand *out, long long maxout, long long *numcands,
                 double *latency_ms)
{
    if (!p) return AB_ERR_ARG;
    std::unique_lock<std::mutex> lk(p->mu);
    auto it = p->reqs.find(ticket);
    if (it == p->reqs.end()) {
        p->err = "unknown ticket";
        return AB_ERR_ARG;
    }
    Request *r = it->second;
    p->cv_done.wait(lk, [&] { return r->done; });
    long long n = (long long) r->cands.size();
    if (numcands) *numcands = n;
    if (latency_ms) *latency_ms = r->t_done - r->t_submit;
    if (r->rc) {
        p->err = r->err;
        int rc = r->rc;
        p->reqs.erase(it);
        delete r;
        return rc;
    }
    if (!out) return AB_OK;                       // count only; the result stays
    for (long long i = 0; i < n && i < maxout; i++) out[i] = r->cands[i];
    if (n > maxout) return AB_ERR_OVERFLOW;
    p->reqs.erase(it);
    delete r;
    return AB_OK;
}

int ab_pool_stats(ab_pool *p, long long *completed, double *p50_ms, double *p99_ms,
                  double *busy_ms)
{
    if (!p) return AB_ERR_ARG;
    std::lock_guard<std::mutex> lk(p->mu);
    std::vector<double> l = p->latencies;
    std::sort(l.begin(), l.end());
    auto pct = [&](double q) {
        if (l.empty()) return 0.0;
        size_t i = (size_t) (q * (double) (l.size() - 1) + 0.5);
        return l[std::min(i, l.size() - 1)];
    };
    if (completed) *completed = p->completed;
    if (p50_ms) *p50_ms = pct(0.50);
    if (p99_ms) *p99_ms = pct(0.99);
    if (busy_ms) *busy_ms = p->busy_first < 0 ? 0.0 : p->busy_last - p->busy_first;
    return AB_OK;
}

int ab_pool_reset_stats(ab_pool *p)
{
    if (!p) return AB_ERR_ARG;
    std::lock_guard<std::mutex> lk(p->mu);
    p->latencies.clear();
    p->completed = 0;
    p->busy_first = -1;
    p->busy_last = 0;
    return AB_OK;
}

}  // extern "C"
