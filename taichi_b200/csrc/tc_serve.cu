// tc_serve.cu -- the served form: resident matrices, admission by HBM
// footprint, and continuous batching of SpMV requests.
//
// No counterpart in the reference (which formats, uploads, multiplies and
// frees one matrix per call, TaiChi.cu:1331-1456).  A tc_server keeps
// admitted plans resident; a request names a plan and carries a host x and a
// host y.  The request loop (tc_server_run) admits requests as they arrive
// and, whenever one of its launch contexts is free, packs every arrived
// request that fits into that context's device arena into one batch: the x
// copies, one multiply launch over all of the batch's tiles (heterogeneous
// matrices, the same tile code as tc_spmv, so each y is bit-identical alone
// and in a mix), and the y copies go on the context's stream.  Several
// contexts are in flight at once, so one batch's copies overlap another's
// multiply.  The plain form multiplies one request at a time.  With
// TC_SERVE_DEVICE_VECTORS the requests' x and y are device vectors that the
// caller owns (no copies; a batch is one launch over the requests' tiles).

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <new>
#include <vector>

#include "tc_internal.h"
#include "tc_tile.cuh"

namespace tc {
namespace {

struct ReqDesc {
    int plan;          // index into the server's device plan table
    int tile_begin;    // first global tile of this request in the batch
    const float *x;
    float *y;
};

constexpr int kMaxBatch = 256;

// One CTA per work item (tile, or quarter of a wide direct tile) of nreq
// requests whose matrices all have plain (SIGNED = false) or all hybrid
// words; request i owns items [reqs[i].tile_begin, reqs[i + 1].tile_begin)
// of the grid.  Thread 0 finds the CTA's request by binary search and parks
// its plan descriptor in shared memory.  LEAN: every admitted plan holds only
// stream, direct and long tiles.
template <bool SIGNED, bool LEAN>
__global__ void __launch_bounds__(kBlock, LEAN ? kItemMinBlocks : 1)
    serve_kernel(const DevPlan *__restrict__ plans, const ReqDesc *__restrict__ reqs, int nreq)
{
    __shared__ DevPlan sp;
    __shared__ ReqDesc sr;
    __shared__ int sitem;
    const int g = blockIdx.x;
    if (threadIdx.x == 0) {
        int lo = 0, hi = nreq;                     // tile_begin[lo] <= g < tile_begin[hi]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (reqs[mid].tile_begin <= g) lo = mid; else hi = mid;
        }
        sr = reqs[lo];
        sp = plans[sr.plan];
        sitem = g - sr.tile_begin;
    }
    __syncthreads();
    const int parts = tile_parts(sp.per_tile);
    const Tile t = sp.tiles[sitem / parts];
    run_tile_part<SIGNED, LEAN>(sp, t, sitem % parts, sr.x, sr.y, false);
}

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace
}  // namespace tc

using tc::fail;

struct tc_server {
    tc_serve_config cfg{};
    struct Ctx {
        cudaStream_t s = nullptr;
        cudaEvent_t done = nullptr;
        float *arena = nullptr;            // device x / y slots
        tc::ReqDesc *h_desc = nullptr;     // pinned
        tc::ReqDesc *d_desc = nullptr;
        std::vector<int> reqs;
        bool busy = false;
    };
    std::vector<Ctx> ctx;
    std::vector<tc_plan *> plans;          // admitted (not owned); null = evicted
    std::vector<int64_t> footprint;
    int64_t used = 0;
    tc::DevPlan *d_plans = nullptr;
    int max_plans = 0;
    int sms = 148;
    int nonlean = 0;                       // admitted plans with lane or merge tiles
};

namespace {
bool lean_plan(const tc_plan *p) { return p->dev_plan().per_tile >= 2; }
}  // namespace

namespace {

int64_t vector_bytes(const tc_plan *p) { return 4LL * ((int64_t)p->N + p->M) + 64; }

}  // namespace

extern "C" {

void tc_serve_config_default(tc_serve_config *c)
{
    if (!c) return;
    c->hbm_budget = 64LL << 30;
    c->arena_bytes = 256LL << 20;
    c->contexts = 6;
    c->max_batch = 64;
    c->max_plans = 1024;
}

tc_status tc_server_create(const tc_serve_config *cfg, tc_server **out)
{
    if (!out) return fail(TC_ERR_INVALID, "tc_server_create: null output");
    *out = nullptr;
    tc_serve_config c;
    tc_serve_config_default(&c);
    if (cfg) c = *cfg;
    if (c.contexts < 1 || c.contexts > 16 || c.max_batch < 1 || c.max_batch > tc::kMaxBatch ||
        c.arena_bytes < 4096 || c.max_plans < 1)
        return fail(TC_ERR_INVALID, "tc_server_create: bad configuration");
    if (c.hbm_budget < c.contexts * c.arena_bytes)
        return fail(TC_ERR_CAPACITY, "HBM budget below the request arenas (%lld < %d x %lld)",
                    (long long)c.hbm_budget, c.contexts, (long long)c.arena_bytes);
    tc_server *sv = new (std::nothrow) tc_server();
    if (!sv) return fail(TC_ERR_ALLOC, "host allocation");
    sv->cfg = c;
    sv->max_plans = c.max_plans;
    sv->used = c.contexts * c.arena_bytes;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sv->sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaMalloc(&sv->d_plans, sizeof(tc::DevPlan) * (size_t)c.max_plans);
    sv->ctx.resize(c.contexts);
    for (auto &x : sv->ctx) {
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&x.s, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&x.done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMalloc(&x.arena, (size_t)c.arena_bytes);
        if (e == cudaSuccess) e = cudaMallocHost(&x.h_desc, sizeof(tc::ReqDesc) * tc::kMaxBatch);
        if (e == cudaSuccess) e = cudaMalloc(&x.d_desc, sizeof(tc::ReqDesc) * tc::kMaxBatch);
    }
    if (e != cudaSuccess) {
        tc_server_destroy(sv);
        return fail(TC_ERR_ALLOC, "server buffers: %s", cudaGetErrorString(e));
    }
    *out = sv;
    return TC_OK;
}

// Admission by HBM footprint: the plan's resident bytes must fit the budget
// left after the arenas and the plans already admitted, and one request's x
// and y must fit an arena.
tc_status tc_server_admit(tc_server *sv, tc_plan *plan, int *id)
{
    if (!sv || !plan || !id) return fail(TC_ERR_INVALID, "tc_server_admit: null argument");
    const int64_t fp = (int64_t)plan->dev_bytes;
    if (vector_bytes(plan) > sv->cfg.arena_bytes)
        return fail(TC_ERR_CAPACITY, "x and y of this matrix (%lld bytes) exceed an arena (%lld)",
                    (long long)vector_bytes(plan), (long long)sv->cfg.arena_bytes);
    if (sv->used + fp > sv->cfg.hbm_budget)
        return fail(TC_ERR_CAPACITY, "HBM budget: %lld used + %lld > %lld", (long long)sv->used,
                    (long long)fp, (long long)sv->cfg.hbm_budget);
    int slot = -1;
    for (size_t i = 0; i < sv->plans.size(); ++i)
        if (!sv->plans[i]) { slot = (int)i; break; }
    if (slot < 0) {
        if ((int)sv->plans.size() >= sv->max_plans) return fail(TC_ERR_CAPACITY, "plan table full");
        slot = (int)sv->plans.size();
        sv->plans.push_back(nullptr);
        sv->footprint.push_back(0);
    }
    const tc::DevPlan dp = plan->dev_plan();
    TC_CUDA(cudaMemcpy(sv->d_plans + slot, &dp, sizeof dp, cudaMemcpyHostToDevice));
    sv->plans[slot] = plan;
    sv->footprint[slot] = fp;
    sv->nonlean += lean_plan(plan) ? 0 : 1;
    sv->used += fp;
    *id = slot;
    return TC_OK;
}

tc_status tc_server_evict(tc_server *sv, int id)
{
    if (!sv || id < 0 || id >= (int)sv->plans.size() || !sv->plans[id])
        return fail(TC_ERR_INVALID, "tc_server_evict: no such matrix");
    sv->used -= sv->footprint[id];
    sv->nonlean -= lean_plan(sv->plans[id]) ? 0 : 1;
    sv->plans[id] = nullptr;
    sv->footprint[id] = 0;
    return TC_OK;
}

int64_t tc_server_hbm_used(const tc_server *sv) { return sv ? sv->used : 0; }

tc_status tc_server_run(tc_server *sv, int nreq, const double *arrival_s, const int *matrix,
                        const float *const *h_x, float *const *h_y, int mode, double *latency_ms,
                        tc_serve_stats *stats)
{
    if (!sv || nreq < 0 || (nreq && (!arrival_s || !matrix || !h_x || !h_y)))
        return fail(TC_ERR_INVALID, "tc_server_run: bad arguments");
    for (int r = 0; r < nreq; ++r)
        if (matrix[r] < 0 || matrix[r] >= (int)sv->plans.size() || !sv->plans[matrix[r]])
            return fail(TC_ERR_INVALID, "request %d names matrix %d, which is not admitted", r, matrix[r]);
    if (mode < 0 || mode > 3) return fail(TC_ERR_INVALID, "tc_server_run: mode %d", mode);
    const bool device_vectors = (mode & TC_SERVE_DEVICE_VECTORS) != 0;
    std::vector<double> done(nreq, 0.0);
    int64_t batches = 0, launched = 0;
    const double t0 = tc::now_s();
    auto slot_floats = [](int64_t n) { return ((n + 63) / 64) * 64; };   // 256-byte slots

    if (mode & 1) {    // plain: one synchronous request at a time
        tc_server::Ctx &c = sv->ctx[0];
        for (int r = 0; r < nreq; ++r) {
            while (tc::now_s() - t0 < arrival_s[r]) { }
            const tc_plan *p = sv->plans[matrix[r]];
            if (device_vectors) {
                TC_CHECK(tc_spmv(p, h_x[r], h_y[r], c.s));
            } else {
                float *dx = c.arena, *dy = c.arena + slot_floats(p->N);
                if (p->N) TC_CUDA(cudaMemcpyAsync(dx, h_x[r], 4 * (size_t)p->N, cudaMemcpyHostToDevice, c.s));
                TC_CHECK(tc_spmv(p, dx, dy, c.s));
                if (p->M) TC_CUDA(cudaMemcpyAsync(h_y[r], dy, 4 * (size_t)p->M, cudaMemcpyDeviceToHost, c.s));
            }
            TC_CUDA(cudaStreamSynchronize(c.s));
            done[r] = tc::now_s() - t0;
            ++batches;
        }
    } else {           // continuous batching over the launch contexts
        std::deque<int> pending;
        std::vector<tc::ReqDesc> batch;    // the batch being packed, arrival order
        std::vector<int> order;            // its request indices
        int next = 0, completed = 0;
        while (completed < nreq) {
            const double now = tc::now_s() - t0;
            while (next < nreq && arrival_s[next] <= now) pending.push_back(next++);
            for (auto &c : sv->ctx) {
                if (!c.busy) continue;
                const cudaError_t q = cudaEventQuery(c.done);
                if (q == cudaErrorNotReady) continue;
                if (q != cudaSuccess) return fail(TC_ERR_CUDA, "batch failed: %s", cudaGetErrorString(q));
                const double t = tc::now_s() - t0;
                for (int r : c.reqs) done[r] = t;
                completed += (int)c.reqs.size();
                c.reqs.clear();
                c.busy = false;
            }
            if (pending.empty()) continue;
            tc_server::Ctx *free_ctx = nullptr;
            for (auto &c : sv->ctx)
                if (!c.busy) { free_ctx = &c; break; }
            if (!free_ctx) continue;
            tc_server::Ctx &c = *free_ctx;
            // pack arrived requests into the arena
            int64_t used = 0;
            int nb = 0;
            batch.clear();
            order.clear();
            while (!pending.empty() && nb < sv->cfg.max_batch) {
                const int r = pending.front();
                const tc_plan *p = sv->plans[matrix[r]];
                if (device_vectors) {   // the request's own device x and y
                    batch.push_back(tc::ReqDesc{matrix[r], 0, h_x[r], h_y[r]});
                } else {                // x and y slots in the context's arena
                    const int64_t need = slot_floats(p->N) + slot_floats(p->M);
                    if ((used + need) * 4 > sv->cfg.arena_bytes) break;
                    float *dx = c.arena + used, *dy = dx + slot_floats(p->N);
                    used += need;
                    batch.push_back(tc::ReqDesc{matrix[r], 0, dx, dy});
                    if (p->N) TC_CUDA(cudaMemcpyAsync(dx, h_x[r], 4 * (size_t)p->N, cudaMemcpyHostToDevice, c.s));
                }
                order.push_back(r);
                pending.pop_front();
                ++nb;
            }
            // plain matrices' requests first, then hybrid ones: one launch each,
            // one CTA per tile, tiles numbered from 0 within each launch
            int np = 0, tiles[2] = {0, 0};
            for (int pass = 0, k = 0; pass < 2; ++pass)
                for (int i = 0; i < nb; ++i) {
                    const tc_plan *p = sv->plans[batch[i].plan];
                    if (p->hybrid != pass) continue;
                    c.h_desc[k] = batch[i];
                    c.h_desc[k].tile_begin = tiles[pass];
                    tiles[pass] += p->ntiles * tc::tile_parts(p->dev_plan().per_tile);
                    c.reqs.push_back(order[i]);
                    np += pass == 0;
                    ++k;
                }
            TC_CUDA(cudaMemcpyAsync(c.d_desc, c.h_desc, sizeof(tc::ReqDesc) * nb, cudaMemcpyHostToDevice, c.s));
            const bool lean = sv->nonlean == 0;
            if (tiles[0] > 0) {
                if (lean) tc::serve_kernel<false, true><<<tiles[0], tc::kBlock, 0, c.s>>>(sv->d_plans, c.d_desc, np);
                else tc::serve_kernel<false, false><<<tiles[0], tc::kBlock, 0, c.s>>>(sv->d_plans, c.d_desc, np);
            }
            if (tiles[1] > 0) {
                const tc::ReqDesc *hd = c.d_desc + np;
                if (lean) tc::serve_kernel<true, true><<<tiles[1], tc::kBlock, 0, c.s>>>(sv->d_plans, hd, nb - np);
                else tc::serve_kernel<true, false><<<tiles[1], tc::kBlock, 0, c.s>>>(sv->d_plans, hd, nb - np);
            }
            TC_CUDA(cudaGetLastError());
            for (int i = 0; i < nb && !device_vectors; ++i) {
                const int r = c.reqs[i];
                const tc_plan *p = sv->plans[matrix[r]];
                if (p->M) TC_CUDA(cudaMemcpyAsync(h_y[r], c.h_desc[i].y, 4 * (size_t)p->M, cudaMemcpyDeviceToHost, c.s));
            }
            TC_CUDA(cudaEventRecord(c.done, c.s));
            c.busy = true;
            ++batches;
            launched += nb;
        }
    }
    // statistics
    std::vector<double> lat(nreq);
    double first = nreq ? arrival_s[0] : 0.0, last = 0.0;
    for (int r = 0; r < nreq; ++r) {
        lat[r] = 1e3 * (done[r] - arrival_s[r]);
        if (latency_ms) latency_ms[r] = lat[r];
        first = std::min(first, arrival_s[r]);
        last = std::max(last, done[r]);
    }
    if (stats) {
        memset(stats, 0, sizeof *stats);
        stats->requests = nreq;
        stats->batches = batches;
        stats->seconds = last - first;
        stats->spmv_per_s = stats->seconds > 0 ? nreq / stats->seconds : 0.0;
        std::vector<double> s = lat;
        std::sort(s.begin(), s.end());
        if (nreq) {
            auto pct = [&](double q) { return s[std::min<size_t>(s.size() - 1, (size_t)(q * (s.size() - 1) + 0.5))]; };
            stats->p50_ms = pct(0.50);
            stats->p99_ms = pct(0.99);
            stats->max_ms = s.back();
            double sum = 0;
            for (double v : s) sum += v;
            stats->mean_ms = sum / nreq;
        }
        stats->mean_batch = batches ? (double)nreq / batches : 0.0;
    }
    return TC_OK;
}

tc_status tc_server_destroy(tc_server *sv)
{
    if (!sv) return TC_OK;
    for (auto &c : sv->ctx) {
        if (c.s) cudaStreamSynchronize(c.s);
        if (c.arena) cudaFree(c.arena);
        if (c.d_desc) cudaFree(c.d_desc);
        if (c.h_desc) cudaFreeHost(c.h_desc);
        if (c.done) cudaEventDestroy(c.done);
        if (c.s) cudaStreamDestroy(c.s);
    }
    if (sv->d_plans) cudaFree(sv->d_plans);
    delete sv;
    return TC_OK;
}

}  // extern "C"
