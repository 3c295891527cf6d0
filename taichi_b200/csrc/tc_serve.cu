// tc_serve.cu -- the served form: resident matrices, admission by HBM
// footprint, and continuous batching of SpMV requests.
//
// No counterpart in the reference (which formats, uploads, multiplies and
// frees one matrix per call, TaiChi.cu:1331-1456).  A tc_server keeps
// admitted plans resident.  Requests (a matrix id, an x and a y) are
// submitted from any thread (tc_server_submit) and completed by the
// server's dispatcher thread: whenever fewer than `max_inflight` batches are
// on the GPU and requests are waiting, it packs every waiting request (up to
// max_batch, and, for host vectors, what fits the context's device arena)
// into one batch on a free launch context -- the x copies, one multiply
// launch over all of the batch's tiles (heterogeneous matrices, the same
// tile code as tc_spmv, so each y is bit-identical alone and in a mix), the
// y copies -- and records an event.  So the batch size
// follows the load: at a low rate every request launches at once; at a high
// rate the requests that arrive while batches run are taken together by the
// next one.  Completion is polled per context; a request's completion time
// is when the dispatcher sees its batch's event.  tc_server_run replays a
// timed request trace through the same path (or, in the plain form, one
// synchronous request at a time on the calling thread).

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "tc_internal.h"
#include "tc_tile.cuh"

namespace tc {
namespace {

struct ReqDesc {
    int plan;          // index into the server's device plan table
    int tile_begin;    // first work item of this request in its launch
    const float *x;
    float *y;
};

constexpr int kMaxBatch = 128;

// A batch's request list, passed by value as the kernel's parameter (no
// descriptor copy before the launch).
struct BatchArgs {
    int n;
    ReqDesc r[kMaxBatch];
};

// One CTA per work item (tile, or quarter of a wide direct tile) of the
// batch's requests; request i owns items [r[i].tile_begin, r[i + 1].tile_begin).
// Thread 0 finds the CTA's request by binary search and parks its plan
// descriptor in shared memory; the CTA then runs the tile code of its plan's
// word kind (plain or hybrid), so one launch serves every request of the
// batch.  LEAN: every admitted plan holds only stream, direct and long tiles.
template <bool LEAN>
__global__ void __launch_bounds__(kBlock, LEAN ? kItemMinBlocks : 1)
    serve_kernel(const DevPlan *__restrict__ plans, const __grid_constant__ BatchArgs b)
{
    __shared__ DevPlan sp;
    __shared__ ReqDesc sr;
    __shared__ int sitem;
    const int g = blockIdx.x;
    if (threadIdx.x == 0) {
        int lo = 0, hi = b.n;                      // r[lo].tile_begin <= g < r[hi].tile_begin
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (b.r[mid].tile_begin <= g) lo = mid; else hi = mid;
        }
        sr = b.r[lo];
        sp = plans[sr.plan];
        sitem = g - sr.tile_begin;
    }
    __syncthreads();
    const int parts = tile_parts(sp.per_tile);
    const Tile t = sp.tiles[sitem / parts];
    if (sp.hybrid) run_tile_part<true, LEAN>(sp, t, sitem % parts, sr.x, sr.y, false);
    else run_tile_part<false, LEAN>(sp, t, sitem % parts, sr.x, sr.y, false);
}

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

enum SlotState : int { kFree = 0, kQueued = 1, kRunning = 2, kDone = 3, kFailed = 4 };

}  // namespace
}  // namespace tc

using tc::fail;

struct tc_server {
    tc_serve_config cfg{};
    struct Ctx {
        cudaStream_t s = nullptr;
        cudaEvent_t done = nullptr;
        cudaStream_t s2 = nullptr;          // large requests' own launches, beside the batch launch
        cudaEvent_t fork = nullptr, join = nullptr;
        float *arena = nullptr;            // device x / y slots (host-vector requests)
        std::vector<uint64_t> reqs;        // tickets of the batch in flight
        bool busy = false;
        double t_launch = 0.0;             // when its batch was launched
    };
    std::vector<Ctx> ctx;
    std::vector<tc_plan *> plans;          // admitted (not owned); null = evicted
    std::vector<int64_t> footprint;
    std::vector<int> inflight;             // queued or running requests per plan
    int64_t used = 0;
    tc::DevPlan *d_plans = nullptr;
    int max_plans = 0;
    int nonlean = 0;                       // admitted plans with lane or merge tiles
    std::mutex admit_mu;                   // plan table vs. the dispatcher

    // online requests: a ring of slots, slot = ticket mod capacity
    struct Slot {
        std::atomic<int> state{tc::kFree};
        uint64_t ticket = 0;
        int matrix = 0;
        const float *x = nullptr;
        float *y = nullptr;
        double t_submit = 0.0, t_done = 0.0;
        double *done_out = nullptr;        // optional: where the completion time goes
    };
    Slot *slots = nullptr;
    uint64_t ring = 0;                     // capacity (power of two)
    std::mutex q_mu;
    std::deque<uint64_t> submitted;        // tickets waiting for the dispatcher
    std::atomic<uint64_t> next_ticket{1};
    std::thread worker;
    std::atomic<bool> running{false}, stop{false};
    std::atomic<int> worker_status{TC_OK};
    int mode_device_vectors = 0;
    // statistics since start
    std::mutex st_mu;
    std::vector<double> lat_ms;
    int64_t batches = 0, completed = 0;
    double t_first = 0.0, t_last = 0.0;
    double service_s = 0.0, launch_s = 0.0;   // summed over batches: launch -> seen done, host packing
    std::string worker_error;
};

namespace {

bool lean_plan(const tc_plan *p) { return p->dev_plan().per_tile >= 2; }
int64_t slot_floats(int64_t n) { return ((n + 63) / 64) * 64; }   // 256-byte slots
// arena bytes of one host-vector request's x and y slots
int64_t vector_bytes(const tc_plan *p) { return 4 * (slot_floats(p->N) + slot_floats(p->M)); }

// Marks the requests of a finished context done at time t.
void complete_ctx(tc_server *sv, tc_server::Ctx &c, double t, bool ok)
{
    std::lock_guard<std::mutex> lk(sv->st_mu);
    for (uint64_t tk : c.reqs) {
        tc_server::Slot &s = sv->slots[tk & (sv->ring - 1)];
        s.t_done = t;
        if (s.done_out) *s.done_out = t;
        sv->lat_ms.push_back(1e3 * (t - s.t_submit));
        sv->t_last = std::max(sv->t_last, t);
        __atomic_fetch_sub(&sv->inflight[s.matrix], 1, __ATOMIC_RELAXED);
        s.state.store(ok ? tc::kDone : tc::kFailed, std::memory_order_release);
    }
    sv->completed += (int64_t)c.reqs.size();
    sv->service_s += t - c.t_launch;
    c.reqs.clear();
    c.busy = false;
}

// Packs waiting requests (front of `pending`) into one batch on context c
// and launches it.  Returns the number of requests taken.
tc_status launch_batch(tc_server *sv, tc_server::Ctx &c, std::deque<uint64_t> &pending, int *taken)
{
    *taken = 0;
    const bool dv = sv->mode_device_vectors != 0;
    tc::BatchArgs args;
    args.n = 0;
    int tiles = 0;
    int64_t used = 0;
    std::vector<std::pair<uint64_t, int>> order;    // ticket, 0: shared launch, 1: its own
    std::vector<tc::ReqDesc> solo;
    c.reqs.clear();                                 // every request taken, so a failure can fail them
    while (!pending.empty() && (int)order.size() < sv->cfg.max_batch) {
        const uint64_t tk = pending.front();
        tc_server::Slot &s = sv->slots[tk & (sv->ring - 1)];
        const tc_plan *p = sv->plans[s.matrix];
        const float *dx = s.x;
        float *dy = s.y;
        if (!dv) {                                     // x and y slots in the context's arena
            const int64_t need = slot_floats(p->N) + slot_floats(p->M);
            if ((used + need) * 4 > sv->cfg.arena_bytes) break;
            float *ax = c.arena + used;
            dy = ax + slot_floats(p->N);
            dx = ax;
            used += need;
            if (p->N) TC_CUDA(cudaMemcpyAsync(ax, s.x, 4 * (size_t)p->N, cudaMemcpyHostToDevice, c.s));
        }
        if (sv->cfg.solo_bytes > 0 && p->spmv_bytes() >= sv->cfg.solo_bytes) {
            // a large matrix runs its own multiply kernel (the one tc_spmv
            // launches) on the context's second stream, beside the batch launch
            solo.push_back(tc::ReqDesc{s.matrix, 0, dx, dy});
            order.emplace_back(tk, 1);
        } else {
            args.r[args.n] = tc::ReqDesc{s.matrix, tiles, dx, dy};
            tiles += p->ntiles * tc::tile_parts(p->dev_plan().per_tile);
            ++args.n;
            order.emplace_back(tk, 0);
        }
        s.state.store(tc::kRunning, std::memory_order_relaxed);
        c.reqs.push_back(tk);
        pending.pop_front();
    }
    if (order.empty()) return TC_OK;
    if (!solo.empty()) {                           // after the x copies
        TC_CUDA(cudaEventRecord(c.fork, c.s));
        TC_CUDA(cudaStreamWaitEvent(c.s2, c.fork, 0));
        for (const tc::ReqDesc &d : solo) TC_CHECK(tc::launch_plan(sv->plans[d.plan], d.x, d.y, c.s2));
        TC_CUDA(cudaEventRecord(c.join, c.s2));
    }
    const bool lean = sv->nonlean == 0;
    if (tiles > 0) {
        if (lean) tc::serve_kernel<true><<<tiles, tc::kBlock, 0, c.s>>>(sv->d_plans, args);
        else tc::serve_kernel<false><<<tiles, tc::kBlock, 0, c.s>>>(sv->d_plans, args);
    }
    TC_CUDA(cudaGetLastError());
    if (!solo.empty()) TC_CUDA(cudaStreamWaitEvent(c.s, c.join, 0));
    if (!dv) {
        int k[2] = {0, 0};
        for (auto &o : order) {
            const tc_server::Slot &s = sv->slots[o.first & (sv->ring - 1)];
            const tc_plan *p = sv->plans[s.matrix];
            const tc::ReqDesc &d = o.second == 1 ? solo[k[1]++] : args.r[k[0]++];
            if (p->M) TC_CUDA(cudaMemcpyAsync(s.y, d.y, 4 * (size_t)p->M, cudaMemcpyDeviceToHost, c.s));
        }
    }
    TC_CUDA(cudaEventRecord(c.done, c.s));
    c.busy = true;
    *taken = (int)order.size();
    return TC_OK;
}

// The dispatcher: reaps finished batches, takes submitted requests, and
// launches a batch whenever fewer than max_inflight are on the GPU.
void dispatcher(tc_server *sv, int device)
{
    cudaSetDevice(device);
    std::deque<uint64_t> pending;
    int busy = 0;
    for (;;) {
        bool idle = true;
        for (auto &c : sv->ctx) {                       // reap
            if (!c.busy) continue;
            const cudaError_t q = cudaEventQuery(c.done);
            if (q == cudaErrorNotReady) continue;
            const double t = tc::now_s();
            if (q != cudaSuccess) {
                std::lock_guard<std::mutex> lk(sv->st_mu);
                sv->worker_error = cudaGetErrorString(q);
                sv->worker_status.store(TC_ERR_CUDA);
            }
            complete_ctx(sv, c, t, q == cudaSuccess);
            --busy;
            idle = false;
        }
        {                                               // intake
            std::lock_guard<std::mutex> lk(sv->q_mu);
            while (!sv->submitted.empty()) {
                pending.push_back(sv->submitted.front());
                sv->submitted.pop_front();
            }
        }
        while (!pending.empty() && busy < sv->cfg.max_inflight) {   // launch
            tc_server::Ctx *fc = nullptr;
            for (auto &c : sv->ctx)
                if (!c.busy) { fc = &c; break; }
            if (!fc) break;
            int taken = 0;
            const double tl = tc::now_s();
            const tc_status st = launch_batch(sv, *fc, pending, &taken);
            fc->t_launch = tl;
            if (st != TC_OK) {                           // the requests it took fail
                {
                    std::lock_guard<std::mutex> lk(sv->st_mu);
                    sv->worker_error = tc_last_error();
                }
                sv->worker_status.store(st);
                cudaStreamSynchronize(fc->s);                // nothing of it stays in flight
                cudaStreamSynchronize(fc->s2);
                complete_ctx(sv, *fc, tc::now_s(), false);
                break;
            }
            if (taken == 0) break;                      // (cannot happen: one request always fits)
            ++busy;
            {
                std::lock_guard<std::mutex> lk(sv->st_mu);
                ++sv->batches;
                sv->launch_s += tc::now_s() - tl;
            }
            idle = false;
        }
        if (sv->worker_status.load() != TC_OK) {        // fail what is left
            const double t = tc::now_s();
            for (auto &c : sv->ctx)
                if (c.busy) {
                    cudaEventSynchronize(c.done);
                    complete_ctx(sv, c, t, false);
                }
            busy = 0;
            for (uint64_t tk : pending) {
                tc_server::Slot &s = sv->slots[tk & (sv->ring - 1)];
                __atomic_fetch_sub(&sv->inflight[s.matrix], 1, __ATOMIC_RELAXED);
                s.state.store(tc::kFailed, std::memory_order_release);
            }
            pending.clear();
        }
        if (sv->stop.load(std::memory_order_acquire) && pending.empty() && busy == 0) {
            std::lock_guard<std::mutex> lk(sv->q_mu);
            if (sv->submitted.empty()) break;
        }
        if (idle) std::this_thread::yield();
    }
}

}  // namespace

extern "C" {

void tc_serve_config_default(tc_serve_config *c)
{
    if (!c) return;
    c->hbm_budget = 64LL << 30;
    c->arena_bytes = 256LL << 20;
    c->contexts = 4;
    c->max_batch = 64;
    c->max_plans = 1024;
    c->max_inflight = 2;
    c->max_pending = 1 << 16;
    c->solo_bytes = 16LL << 20;
}

tc_status tc_server_create(const tc_serve_config *cfg, tc_server **out)
{
    if (!out) return fail(TC_ERR_INVALID, "tc_server_create: null output");
    *out = nullptr;
    tc_serve_config c;
    tc_serve_config_default(&c);
    if (cfg) c = *cfg;
    if (c.contexts < 1 || c.contexts > 16 || c.max_batch < 1 || c.max_batch > tc::kMaxBatch ||
        c.arena_bytes < 4096 || c.max_plans < 1 || c.max_inflight < 1 || c.max_inflight > c.contexts ||
        c.max_pending < 1 || c.max_pending > (1 << 24))
        return fail(TC_ERR_INVALID, "tc_server_create: bad configuration");
    if (c.hbm_budget < c.contexts * c.arena_bytes)
        return fail(TC_ERR_CAPACITY, "HBM budget below the request arenas (%lld < %d x %lld)",
                    (long long)c.hbm_budget, c.contexts, (long long)c.arena_bytes);
    tc_server *sv = new (std::nothrow) tc_server();
    if (!sv) return fail(TC_ERR_ALLOC, "host allocation");
    sv->cfg = c;
    sv->max_plans = c.max_plans;
    sv->used = c.contexts * c.arena_bytes;
    uint64_t ring = 1;
    while (ring < (uint64_t)c.max_pending) ring <<= 1;
    sv->ring = ring;
    sv->slots = new (std::nothrow) tc_server::Slot[ring];
    if (!sv->slots) {
        delete sv;
        return fail(TC_ERR_ALLOC, "host allocation of %llu request slots", (unsigned long long)ring);
    }
    cudaError_t e = cudaMalloc(&sv->d_plans, sizeof(tc::DevPlan) * (size_t)c.max_plans);
    sv->ctx.resize(c.contexts);
    for (auto &x : sv->ctx) {
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&x.s, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&x.done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&x.s2, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&x.fork, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&x.join, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMalloc(&x.arena, (size_t)c.arena_bytes);
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
    std::lock_guard<std::mutex> lk(sv->admit_mu);
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
        if (sv->running.load()) return fail(TC_ERR_UNSUPPORTED, "the plan table grows only while the server is stopped");
        slot = (int)sv->plans.size();
        sv->plans.push_back(nullptr);
        sv->footprint.push_back(0);
        sv->inflight.push_back(0);
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
    if (!sv) return fail(TC_ERR_INVALID, "tc_server_evict: null server");
    std::lock_guard<std::mutex> lk(sv->admit_mu);
    if (id < 0 || id >= (int)sv->plans.size() || !sv->plans[id])
        return fail(TC_ERR_INVALID, "tc_server_evict: no such matrix");
    if (__atomic_load_n(&sv->inflight[id], __ATOMIC_ACQUIRE) > 0)
        return fail(TC_ERR_CAPACITY, "matrix %d has requests in flight", id);
    sv->used -= sv->footprint[id];
    sv->nonlean -= lean_plan(sv->plans[id]) ? 0 : 1;
    sv->plans[id] = nullptr;
    sv->footprint[id] = 0;
    return TC_OK;
}

int64_t tc_server_hbm_used(const tc_server *sv) { return sv ? sv->used : 0; }

tc_status tc_server_start(tc_server *sv, int device_vectors)
{
    if (!sv) return fail(TC_ERR_INVALID, "tc_server_start: null server");
    if (sv->running.load()) return fail(TC_ERR_INVALID, "tc_server_start: already running");
    int dev = 0;
    TC_CUDA(cudaGetDevice(&dev));
    sv->mode_device_vectors = device_vectors ? 1 : 0;
    sv->stop.store(false);
    sv->worker_status.store(TC_OK);
    sv->worker_error.clear();
    {
        std::lock_guard<std::mutex> lk(sv->st_mu);
        sv->lat_ms.clear();
        sv->batches = sv->completed = 0;
        sv->t_first = sv->t_last = 0.0;
        sv->service_s = sv->launch_s = 0.0;
    }
    sv->running.store(true);
    try {
        sv->worker = std::thread(dispatcher, sv, dev);
    } catch (...) {
        sv->running.store(false);
        return fail(TC_ERR_ALLOC, "could not start the dispatcher thread");
    }
    return TC_OK;
}

}  // extern "C"

// Queues one request; `done_out` (optional) receives its completion time.
static tc_status submit_impl(tc_server *sv, int matrix_id, const float *x, float *y, double *done_out,
                             uint64_t *ticket)
{
    if (!sv || !ticket) return fail(TC_ERR_INVALID, "tc_server_submit: null argument");
    if (!sv->running.load() || sv->stop.load()) return fail(TC_ERR_INVALID, "tc_server_submit: server not started");
    {
        std::lock_guard<std::mutex> lk(sv->admit_mu);
        if (matrix_id < 0 || matrix_id >= (int)sv->plans.size() || !sv->plans[matrix_id])
            return fail(TC_ERR_INVALID, "matrix %d is not admitted", matrix_id);
        const tc_plan *p = sv->plans[matrix_id];
        if ((p->N && !x) || (p->M && !y)) return fail(TC_ERR_INVALID, "tc_server_submit: null vector");
        __atomic_fetch_add(&sv->inflight[matrix_id], 1, __ATOMIC_RELAXED);
    }
    std::lock_guard<std::mutex> lk(sv->q_mu);
    const uint64_t tk = sv->next_ticket.load(std::memory_order_relaxed);
    tc_server::Slot &s = sv->slots[tk & (sv->ring - 1)];
    const int st = s.state.load(std::memory_order_acquire);
    if (st == tc::kQueued || st == tc::kRunning) {
        __atomic_fetch_sub(&sv->inflight[matrix_id], 1, __ATOMIC_RELAXED);
        return fail(TC_ERR_CAPACITY, "more than %llu requests outstanding", (unsigned long long)sv->ring);
    }
    sv->next_ticket.store(tk + 1, std::memory_order_release);
    s.ticket = tk;
    s.matrix = matrix_id;
    s.x = x;
    s.y = y;
    s.done_out = done_out;
    s.t_submit = tc::now_s();
    s.state.store(tc::kQueued, std::memory_order_release);
    {
        std::lock_guard<std::mutex> sl(sv->st_mu);
        if (sv->t_first == 0.0) sv->t_first = s.t_submit;
    }
    sv->submitted.push_back(tk);
    *ticket = tk;
    return TC_OK;
}

extern "C" {

tc_status tc_server_submit(tc_server *sv, int matrix_id, const float *x, float *y, uint64_t *ticket)
{
    return submit_impl(sv, matrix_id, x, y, nullptr, ticket);
}

tc_status tc_server_poll(tc_server *sv, uint64_t ticket, int *done)
{
    if (!sv || !done) return fail(TC_ERR_INVALID, "tc_server_poll: null argument");
    *done = 0;
    const tc_server::Slot &s = sv->slots[ticket & (sv->ring - 1)];
    if (ticket == 0 || ticket >= sv->next_ticket.load(std::memory_order_acquire)) return fail(TC_ERR_INVALID, "unknown ticket %llu", (unsigned long long)ticket);
    const int st = s.state.load(std::memory_order_acquire);
    if (s.ticket != ticket) {                  // the slot was reused: this one finished earlier
        *done = 1;
        return TC_OK;
    }
    if (st == tc::kFailed) {
        std::string why;
        {
            std::lock_guard<std::mutex> lk(sv->st_mu);
            why = sv->worker_error;
        }
        const int ws = sv->worker_status.load();
        return fail(ws != TC_OK ? (tc_status)ws : TC_ERR_CUDA, "request %llu failed: %s",
                    (unsigned long long)ticket, why.c_str());
    }
    *done = st == tc::kDone;
    return TC_OK;
}

tc_status tc_server_wait(tc_server *sv, uint64_t ticket, double timeout_s)
{
    const double t0 = tc::now_s();
    for (;;) {
        int done = 0;
        TC_CHECK(tc_server_poll(sv, ticket, &done));
        if (done) return TC_OK;
        if (timeout_s >= 0 && tc::now_s() - t0 > timeout_s)
            return fail(TC_ERR_TIMEOUT, "request %llu not done after %.3f s", (unsigned long long)ticket, timeout_s);
        std::this_thread::yield();
    }
}

static void fill_stats(tc_server *sv, const std::vector<double> &lat, double seconds, int64_t batches,
                       tc_serve_stats *stats, double service_s = 0.0, double launch_s = 0.0)
{
    memset(stats, 0, sizeof *stats);
    const size_t n = lat.size();
    stats->requests = (int64_t)n;
    stats->batches = batches;
    stats->seconds = seconds;
    stats->spmv_per_s = seconds > 0 ? n / seconds : 0.0;
    if (n) {
        std::vector<double> s = lat;
        std::sort(s.begin(), s.end());
        auto pct = [&](double q) { return s[std::min<size_t>(n - 1, (size_t)(q * (n - 1) + 0.5))]; };
        stats->p50_ms = pct(0.50);
        stats->p99_ms = pct(0.99);
        stats->max_ms = s.back();
        double sum = 0;
        for (double v : s) sum += v;
        stats->mean_ms = sum / n;
    }
    stats->mean_batch = batches ? (double)n / batches : 0.0;
    stats->mean_service_ms = batches ? 1e3 * service_s / batches : 0.0;
    stats->mean_launch_us = batches ? 1e6 * launch_s / batches : 0.0;
    (void)sv;
}

tc_status tc_server_stats(tc_server *sv, tc_serve_stats *stats)
{
    if (!sv || !stats) return fail(TC_ERR_INVALID, "tc_server_stats: null argument");
    std::lock_guard<std::mutex> lk(sv->st_mu);
    fill_stats(sv, sv->lat_ms, sv->t_last > sv->t_first ? sv->t_last - sv->t_first : 0.0, sv->batches, stats,
               sv->service_s, sv->launch_s);
    return TC_OK;
}

tc_status tc_server_stop(tc_server *sv)
{
    if (!sv) return fail(TC_ERR_INVALID, "tc_server_stop: null server");
    if (!sv->running.load()) return TC_OK;
    sv->stop.store(true, std::memory_order_release);
    if (sv->worker.joinable()) sv->worker.join();
    sv->running.store(false);
    const int st = sv->worker_status.load();
    return st == TC_OK ? TC_OK : fail((tc_status)st, "dispatcher: %s", sv->worker_error.c_str());   // thread joined
}

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
    if (sv->running.load()) return fail(TC_ERR_INVALID, "tc_server_run: the server is serving online requests");
    const bool device_vectors = (mode & TC_SERVE_DEVICE_VECTORS) != 0;
    std::vector<double> done(nreq, 0.0);
    int64_t batches = 0;
    double t0 = 0.0, service_s = 0.0, launch_s = 0.0;

    if (mode & 1) {    // plain: one synchronous request at a time on this thread
        tc_server::Ctx &c = sv->ctx[0];
        t0 = tc::now_s();
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
    } else {           // continuous batching: submitted at their arrival times
        TC_CHECK(tc_server_start(sv, device_vectors ? 1 : 0));
        std::vector<double> tdone(nreq, 0.0);
        std::vector<uint64_t> tickets(nreq);
        tc_status st = TC_OK;
        t0 = tc::now_s();
        for (int r = 0; r < nreq && st == TC_OK; ++r) {
            while (tc::now_s() - t0 < arrival_s[r]) { }
            st = submit_impl(sv, matrix[r], h_x[r], h_y[r], &tdone[r], &tickets[r]);
        }
        for (int r = 0; r < nreq && st == TC_OK; ++r) st = tc_server_wait(sv, tickets[r], 60.0);
        const tc_status st2 = tc_server_stop(sv);
        TC_CHECK(st);
        TC_CHECK(st2);
        for (int r = 0; r < nreq; ++r) done[r] = tdone[r] > 0 ? tdone[r] - t0 : 0.0;
        std::lock_guard<std::mutex> lk(sv->st_mu);
        batches = sv->batches;
        service_s = sv->service_s;
        launch_s = sv->launch_s;
    }
    // statistics: latency = completion - arrival
    std::vector<double> lat(nreq);
    double first = nreq ? arrival_s[0] : 0.0, last = 0.0;
    for (int r = 0; r < nreq; ++r) {
        lat[r] = 1e3 * (done[r] - arrival_s[r]);
        if (latency_ms) latency_ms[r] = lat[r];
        first = std::min(first, arrival_s[r]);
        last = std::max(last, done[r]);
    }
    if (stats) fill_stats(sv, lat, last - first, batches, stats, service_s, launch_s);
    return TC_OK;
}

tc_status tc_server_destroy(tc_server *sv)
{
    if (!sv) return TC_OK;
    tc_server_stop(sv);
    for (auto &c : sv->ctx) {
        if (c.s) cudaStreamSynchronize(c.s);
        if (c.arena) cudaFree(c.arena);
        if (c.s2) cudaStreamSynchronize(c.s2);
        if (c.done) cudaEventDestroy(c.done);
        if (c.fork) cudaEventDestroy(c.fork);
        if (c.join) cudaEventDestroy(c.join);
        if (c.s2) cudaStreamDestroy(c.s2);
        if (c.s) cudaStreamDestroy(c.s);
    }
    if (sv->d_plans) cudaFree(sv->d_plans);
    delete[] sv->slots;
    delete sv;
    return TC_OK;
}

}  // extern "C"
