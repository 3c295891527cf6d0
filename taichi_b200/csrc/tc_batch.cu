// tc_batch.cu -- many resident plans multiplied in one launch.
//
// The batch flattens the tile lists of all its plans into one work list of
// (plan, tile) pairs -- the plain plans' tiles first, then the hybrid plans'
// -- and runs it with one CTA per work item: one launch for the plain part and
// one for the hybrid part, so each runs tile code of one word kind only.  The
// item's plan descriptor is read once into shared memory.  A CTA per item
// keeps the most independent tiles in flight per SM; a
// persistent grid that walks items in turn serialises each tile's load ->
// gather -> sum chain per CTA and measured slower.  When every plan holds
// only stream, direct and long tiles the lean kernels (no lane-tile code,
// more CTAs per SM) run.  Every tile runs the same device code as the
// single-plan kernel, so each matrix's y is bit-identical alone and inside a
// batch.  The launches are captured once in a CUDA graph and replayed
// (tc_batch_graph_launch).

#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <numeric>

#include "tc_internal.h"
#include "tc_tile.cuh"

namespace tc {
namespace {

struct BatchItem {
    int plan;
    int tile;
    int part;          // quarter of a wide direct tile, else 0
};

// Work items of plain plans (SIGNED = false) or of hybrid plans (true): the
// work list holds the plain plans' items first, and each half runs under
// its own kernel so that neither tile code raises the other's registers.
template <bool SIGNED, bool LEAN>
__global__ void __launch_bounds__(kBlock, LEAN ? kItemMinBlocks : 1)
    batch_kernel(const DevPlan *__restrict__ plans, const BatchItem *__restrict__ items, int nitems,
                 const float *const *xs, float *const *ys)
{
    __shared__ DevPlan sp;                     // the item's plan, read by every thread
    if ((int)blockIdx.x >= nitems) return;     // the grid has one CTA per item
    const BatchItem it = items[blockIdx.x];
    if (threadIdx.x == 0) sp = plans[it.plan];
    __syncthreads();
    const Tile t = sp.tiles[it.tile];
    run_tile_part<SIGNED, LEAN>(sp, t, it.part, xs[it.plan], ys[it.plan], true);
}

}  // namespace
}  // namespace tc

struct tc_batch {
    int n = 0;
    int nitems = 0;
    int nplain = 0;      // items of plain plans (the first ones of the list)
    int grid = 0;
    bool lean = false;
    size_t smem = 0;
    void *dev = nullptr;
    tc::DevPlan *d_plans = nullptr;
    tc::BatchItem *d_items = nullptr;
    const float **d_x = nullptr;
    float **d_y = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

using tc::fail;

extern "C" {

tc_status tc_batch_create(int n, tc_plan *const *plans, const float *const *d_x, float *const *d_y,
                          tc_batch **out)
{
    if (n < 1 || !plans || !d_x || !d_y || !out) return fail(TC_ERR_INVALID, "tc_batch_create: bad arguments");
    *out = nullptr;
    std::vector<tc::DevPlan> dps(n);
    std::vector<tc::BatchItem> items;
    bool lean = true;
    for (int i = 0; i < n; ++i) {
        if (!plans[i]) return fail(TC_ERR_INVALID, "plan %d is null", i);
        dps[i] = plans[i]->dev_plan();
        lean = lean && dps[i].per_tile >= 2;
    }
    for (int pass = 0; pass < 2; ++pass)     // plain plans' items, then hybrid plans'
        for (int i = 0; i < n; ++i)
            if (dps[i].hybrid == pass)
                for (int t = 0; t < dps[i].ntiles; ++t)
                    for (int k = 0; k < tc::tile_parts(dps[i].per_tile); ++k)
                        items.push_back(tc::BatchItem{i, t, k});
    tc_batch *b = new (std::nothrow) tc_batch();
    if (!b) return fail(TC_ERR_ALLOC, "host allocation");
    b->lean = lean;
    b->n = n;
    b->nitems = (int)items.size();
    b->nplain = 0;
    for (const tc::BatchItem &it : items) b->nplain += dps[it.plan].hybrid == 0;
    b->smem = 0;
    size_t o_pl = 0;
    size_t o_it = (sizeof(tc::DevPlan) * n + 255) & ~(size_t)255;
    size_t o_x = o_it + ((sizeof(tc::BatchItem) * items.size() + 255) & ~(size_t)255);
    size_t o_y = o_x + ((sizeof(void *) * n + 255) & ~(size_t)255);
    size_t total = o_y + sizeof(void *) * n + 256;
    char *base = nullptr;
    if (cudaMalloc(&base, total) != cudaSuccess) { delete b; return fail(TC_ERR_ALLOC, "batch tables"); }
    b->dev = base;
    b->d_plans = reinterpret_cast<tc::DevPlan *>(base + o_pl);
    b->d_items = reinterpret_cast<tc::BatchItem *>(base + o_it);
    b->d_x = reinterpret_cast<const float **>(base + o_x);
    b->d_y = reinterpret_cast<float **>(base + o_y);
    cudaError_t e = cudaMemcpy(b->d_plans, dps.data(), sizeof(tc::DevPlan) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !items.empty())
        e = cudaMemcpy(b->d_items, items.data(), sizeof(tc::BatchItem) * items.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_x, d_x, sizeof(void *) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_y, d_y, sizeof(void *) * n, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(base);
        delete b;
        return fail(TC_ERR_CUDA, "tc_batch_create: %s", cudaGetErrorString(e));
    }
    b->grid = std::max(1, b->nitems);                   // one CTA per work item
    *out = b;
    return TC_OK;
}

tc_status tc_batch_run(tc_batch *b, void *stream)
{
    if (!b) return fail(TC_ERR_INVALID, "null batch");
    if (b->nitems == 0) return TC_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const int np = b->nplain, nh = b->nitems - b->nplain;   // one CTA per item
    const tc::BatchItem *hi = b->d_items + np;
    if (b->lean) {
        if (np) tc::batch_kernel<false, true><<<np, tc::kBlock, 0, s>>>(b->d_plans, b->d_items, np, b->d_x, b->d_y);
        if (nh) tc::batch_kernel<true, true><<<nh, tc::kBlock, 0, s>>>(b->d_plans, hi, nh, b->d_x, b->d_y);
    } else {
        if (np) tc::batch_kernel<false, false><<<np, tc::kBlock, 0, s>>>(b->d_plans, b->d_items, np, b->d_x, b->d_y);
        if (nh) tc::batch_kernel<true, false><<<nh, tc::kBlock, 0, s>>>(b->d_plans, hi, nh, b->d_x, b->d_y);
    }
    TC_CUDA(cudaGetLastError());
    return TC_OK;
}

tc_status tc_batch_graph_launch(tc_batch *b, void *stream)
{
    if (!b) return fail(TC_ERR_INVALID, "null batch");
    cudaStream_t s = (cudaStream_t)stream;
    if (!b->exec) {
        cudaStream_t cap;
        TC_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        TC_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        tc_status st = tc_batch_run(b, cap);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(cap, &g);
        cudaStreamDestroy(cap);
        if (st != TC_OK) return st;
        if (e != cudaSuccess) return fail(TC_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
        b->graph = g;
        TC_CUDA(cudaGraphInstantiate(&b->exec, g, 0));
    }
    TC_CUDA(cudaGraphLaunch(b->exec, s));
    return TC_OK;
}

tc_status tc_batch_destroy(tc_batch *b)
{
    if (!b) return TC_OK;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->dev) cudaFree(b->dev);
    delete b;
    return TC_OK;
}

}  // extern "C"
