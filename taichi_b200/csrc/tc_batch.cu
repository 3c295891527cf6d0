// tc_batch.cu -- many resident plans multiplied in one persistent launch.
//
// The batch flattens the tile lists of all its plans into one work list of
// (plan, tile) pairs in plan order and launches one grid of
// (SMs x resident CTAs) CTAs that stride over it.  Every tile runs the same
// device code as the single-plan kernel, so each matrix's y is bit-identical
// alone and inside a batch.  The launch can be captured once in a CUDA graph
// and replayed (tc_batch_graph_launch).

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
};

__global__ void __launch_bounds__(kBlock) batch_kernel(const DevPlan *__restrict__ plans,
                                                       const BatchItem *__restrict__ items,
                                                       int nitems, const float *const *xs,
                                                       float *const *ys)
{
    for (int w = blockIdx.x; w < nitems; w += gridDim.x) {
        const BatchItem it = items[w];
        const DevPlan &p = plans[it.plan];     // read in place (global memory)
        const Tile t = p.tiles[it.tile];
        const float *x = xs[it.plan];
        float *y = ys[it.plan];
        if (p.hybrid) run_tile<true>(p, t, x, y);
        else run_tile<false>(p, t, x, y);
    }
}

}  // namespace
}  // namespace tc

struct tc_batch {
    int n = 0;
    int nitems = 0;
    int grid = 0;
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
    for (int i = 0; i < n; ++i) {
        if (!plans[i]) return fail(TC_ERR_INVALID, "plan %d is null", i);
        dps[i] = plans[i]->dev_plan();
        for (int t = 0; t < dps[i].ntiles; ++t) items.push_back(tc::BatchItem{i, t});
    }
    tc_batch *b = new (std::nothrow) tc_batch();
    if (!b) return fail(TC_ERR_ALLOC, "host allocation");
    b->n = n;
    b->nitems = (int)items.size();
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
    int per_sm = 0, dev = 0, sms = 0;
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tc::batch_kernel, tc::kBlock, b->smem);
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) {
        cudaFree(base);
        delete b;
        return fail(TC_ERR_CUDA, "tc_batch_create: %s", cudaGetErrorString(e));
    }
    b->grid = std::max(1, std::min(b->nitems, std::max(1, per_sm) * sms));
    *out = b;
    return TC_OK;
}

tc_status tc_batch_run(tc_batch *b, void *stream)
{
    if (!b) return fail(TC_ERR_INVALID, "null batch");
    if (b->nitems == 0) return TC_OK;
    tc::batch_kernel<<<b->grid, tc::kBlock, b->smem, (cudaStream_t)stream>>>(
        b->d_plans, b->d_items, b->nitems, b->d_x, b->d_y);
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
