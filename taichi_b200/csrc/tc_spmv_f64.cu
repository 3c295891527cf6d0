// tc_spmv_f64.cu -- the multiply in double precision: y = A x with FP64 x and
// y over the same resident plan (the reference's VALUE_TYPE=double build,
// TaiChi.h:62-64, which turns x, y and the kernels' accumulators into double;
// the pattern and the hybrid format are unchanged).
//
// One 256-thread CTA per tile of the plan's own tile list.  Tiles of short
// rows (stream, direct and one-lane kinds) give each thread whole rows; the
// other kinds (lane, merge tiles) give each warp a row at a time, its lanes
// striding the row's offsets and words, combined by a butterfly; a long row
// (TILE_LONG) gets the whole CTA.  A row adds its dense-diagonal terms in
// offset order, then its CSR words in stored order (signed words of a hybrid
// plan subtract the holes).  The kernel is launched without programmatic
// dependent launch, so x and y follow plain stream order.

#include <cuda_runtime.h>

#include "tc_internal.h"

namespace tc {
namespace {

constexpr int kF64Block = 256;

template <bool SIGNED>
__device__ __forceinline__ double gather64(const double *__restrict__ x, int c)
{
    if (SIGNED) {
        const double v = x[c >> 1];
        return (c & 1) ? v : -v;
    }
    return x[c];
}

// The dense-diagonal terms of row r that lane `lane` of `lanes` owns
// (offsets lane, lane + lanes, ... of each shape holding the row).
__device__ double diag_terms64(const DevPlan &p, const double *__restrict__ x, int r, int lane, int lanes)
{
    double acc = 0.0;
    if (r < p.row_start || r >= p.row_stop) return acc;
    for (int s = 0; s < p.dia_shapes; ++s) {
        const int4 sh = p.shapes[s];
        if (r < sh.x || r >= sh.y) continue;
        const int2 dr = p.shape_dias[s];
        const int cb = r - sh.x + sh.z;
        for (int d = dr.x + lane; d < dr.y; d += lanes) {
            const int c = cb + p.offsets[d];
            if (c >= sh.z && c < sh.z + sh.w) acc += x[c];
        }
    }
    return acc;
}

__device__ __forceinline__ double warp_sum64(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <bool SIGNED>
__global__ void __launch_bounds__(kF64Block) spmv_f64_kernel(DevPlan p, const double *__restrict__ x,
                                                            double *__restrict__ y)
{
    __shared__ double red[kF64Block / 32];
    const Tile t = p.tiles[blockIdx.x];
    const int nr = tile_nrows(t), kind = tile_kind(t);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (kind == TILE_LONG) {
        const int r = t.row0;
        double acc = diag_terms64(p, x, r, threadIdx.x, kF64Block);
        for (int j = p.rowptr[r] + threadIdx.x; j < p.rowptr[r + 1]; j += kF64Block)
            acc += gather64<SIGNED>(x, p.cols[j]);
        acc = warp_sum64(acc);
        if (lane == 0) red[warp] = acc;
        __syncthreads();
        if (warp == 0) {
            double v = lane < kF64Block / 32 ? red[lane] : 0.0;
            v = warp_sum64(v);
            if (lane == 0) y[r] = v;
        }
        return;
    }
    const bool thread_rows = kind == TILE_L1 || kind == TILE_STREAM || kind == TILE_STREAM4 ||
                             kind == TILE_DIRECT4 || kind == TILE_DIRECT_WIDE;
    if (thread_rows) {
        for (int rl = threadIdx.x; rl < nr; rl += kF64Block) {
            const int r = t.row0 + rl;
            double acc = diag_terms64(p, x, r, 0, 1);
            for (int j = p.rowptr[r]; j < p.rowptr[r + 1]; ++j) acc += gather64<SIGNED>(x, p.cols[j]);
            y[r] = acc;
        }
        return;
    }
    for (int rl = warp; rl < nr; rl += kF64Block / 32) {      // lane and merge tiles: a warp per row
        const int r = t.row0 + rl;
        double acc = diag_terms64(p, x, r, lane, 32);
        for (int j = p.rowptr[r] + lane; j < p.rowptr[r + 1]; j += 32) acc += gather64<SIGNED>(x, p.cols[j]);
        acc = warp_sum64(acc);
        if (lane == 0) y[r] = acc;
    }
}

}  // namespace
}  // namespace tc

tc_status tc_spmv_f64(const tc_plan *p, const double *d_x, double *d_y, void *stream)
{
    using namespace tc;
    if (!p || (!d_x && p->N) || (!d_y && p->M)) return fail(TC_ERR_INVALID, "tc_spmv_f64: null argument");
    const DevPlan dp = p->dev_plan();
    if (dp.M == 0 || dp.ntiles == 0) return TC_OK;
    cudaStream_t s = (cudaStream_t)stream;
    if (dp.hybrid) spmv_f64_kernel<true><<<dp.ntiles, kF64Block, 0, s>>>(dp, d_x, d_y);
    else spmv_f64_kernel<false><<<dp.ntiles, kF64Block, 0, s>>>(dp, d_x, d_y);
    TC_CUDA(cudaGetLastError());
    return TC_OK;
}
