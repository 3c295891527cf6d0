// tc_window.cu -- the diagonal-segment multiply: x streamed through shared
// memory in contiguous windows.
//
// In the hybrid format a dense diagonal of a shape reads x at column
// r - xStart + yStart + off for consecutive rows r (TaiChi.cu:1014-1023), so
// the rows [r0, r0 + n) of a tile read one contiguous segment of x per
// offset; on banded and mesh-like matrices the CSR remainder's columns also
// stay within a fixed distance of the row.  A window plan cuts the rows into
// window tiles and gives each tile the x segment [r0 + wlo, r0 + n + whi)
// that covers those columns (wlo / whi chosen per plan from a histogram of
// column - row over all the matrix's accesses).  The multiply is a
// persistent grid, one CTA per SM, with a pipeline of kWinMaxStages stages:
// for each tile the TMA engine copies the row pointers, the CSR words and the
// x window into a stage with three bulk copies (cp.async.bulk, completion on
// an mbarrier), while the CTA sums the rows of the tile staged before it.
// Each thread sums one row at a time: dense-diagonal terms in offset order,
// then the CSR words in stored order, each term read from the staged window
// when its column lies inside it and from global memory otherwise -- the
// terms and order of the one-row-per-thread tiles in tc_tile.cuh, so y is
// bit-identical to the other multiply kernels (and to the batch and served
// launches, which run the plan's ordinary tile list).
//
// Row pointers and CSR words are immutable plan data, copied before
// griddepcontrol.wait; the x windows are copied after it.  Every wait on a
// stage is bounded in time; a give-up sets the plan's error word, waits
// (bounded) for the copies still in flight and returns.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <vector>

#include "tc_internal.h"
#include "tc_tile.cuh"
#include "tc_tma.cuh"

namespace tc {
namespace {

// x bounds of the window of rows [row0, row0 + nr): 16-byte aligned, inside
// the whole float4s of x; empty when x itself is not 16-byte aligned.
__device__ __forceinline__ void win_bounds(const DevPlan &p, int row0, int nr, bool xa, int &wa, int &wlen)
{
    wa = 0;
    wlen = 0;
    if (!xa) return;
    const long n4 = (long)p.N & ~3L;
    const long a = std::max(0L, (long)row0 + p.wlo) & ~3L;
    const long b = std::min(n4, ((long)row0 + nr + p.whi + 3) & ~3L);
    if (b > a) {
        wa = (int)a;
        wlen = (int)std::min<long>(b - a, p.w_xw);
    }
}

// Thread 0: the copies of tile t's row pointers and CSR words into stage
// `st` (the first of the stage barrier's two arrivals).
__device__ __forceinline__ void win_issue_index(const DevPlan &p, const Tile &t, int *st, uint64_t *bar)
{
    const int nr = tile_nrows(t);
    const Window wr = window_of(t.row0, (long)t.row0 + nr + 1);
    const Window wc = window_of(t.nz0, (long)t.nz0 + t.nnz);
    const unsigned br = (unsigned)(wr.b - wr.a), bc = t.nnz ? (unsigned)(wc.b - wc.a) : 0u;
    mbar_expect_tx(bar, br + bc);
    bulk_load(st, reinterpret_cast<const char *>(p.rowptr) + wr.a, br, bar);
    if (bc) bulk_load(st + p.w_rp, reinterpret_cast<const char *>(p.cols) + wc.a, bc, bar);
}

// Thread 0: the copy of tile t's x window (the second arrival).
__device__ __forceinline__ void win_issue_x(const DevPlan &p, const Tile &t, int *st, uint64_t *bar,
                                            const float *x, bool xa)
{
    int wa, wlen;
    win_bounds(p, t.row0, tile_nrows(t), xa, wa, wlen);
    mbar_expect_tx(bar, 4u * (unsigned)wlen);
    if (wlen) bulk_load(st + p.w_rp + p.w_cw, x + wa, 4u * (unsigned)wlen, bar);
}

// A coherent load of x that the compiler may not execute speculatively: the
// global read of an out-of-window column must stay on its branch (a load
// the compiler takes for side-effect free may be if-converted and issued for
// every term, window hits included).
__device__ __forceinline__ float ldx_guarded(const float *p)
{
    float v;
    asm volatile("ld.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
    return v;
}

// x[c] from the staged window when c lies in it, else from global memory.
struct WinX {
    const float *xw;
    const float *x;
    int wa;
    unsigned wlen;
    __device__ __forceinline__ float operator()(int c) const
    {
        const unsigned k = (unsigned)(c - wa);
        if (k < wlen) return xw[k];
        return ldx_guarded(x + c);
    }
};

// Dense-diagonal terms of row r in offset order (diag_row's terms and order).
__device__ __forceinline__ float win_diag_general(const DevPlan &p, const WinX &xv, int r)
{
    float acc = 0.f;
    if (r < p.row_start || r >= p.row_stop) return acc;
    for (int s = 0; s < p.dia_shapes; ++s) {
        const int4 sh = __ldg(p.shapes + s);
        if (r < sh.x || r >= sh.y) continue;
        const int2 dr = __ldg(p.shape_dias + s);
        const int cb = r - sh.x + sh.z;
        for (int d = dr.x; d < dr.y; ++d) {
            const int c = cb + __ldg(p.offsets + d);
            if (c >= sh.z && c < sh.z + sh.w) acc += xv(c);
        }
    }
    return acc;
}

template <bool SIGNED>
__device__ __forceinline__ void win_tile(const DevPlan &p, const Tile &t, const int *st, const float *x,
                                         float *__restrict__ y, bool xa)
{
    const int nr = tile_nrows(t), row0 = t.row0, dc = tile_dclass(t);
    const int *rp = st + window_of(row0, 0).shift;                 // rp[k] = rowptr[row0 + k]
    const int *cw = st + p.w_rp + window_of(t.nz0, 0).shift;       // cw[j] = cols[nz0 + j]
    int wa, wlen;
    win_bounds(p, row0, nr, xa, wa, wlen);
    const WinX xv{reinterpret_cast<const float *>(st + p.w_rp + p.w_cw), x, wa, (unsigned)wlen};
    int2 dr = make_int2(0, 0);
    int cb0 = 0;
    if (SIGNED && dc != kDiagNone && dc != kDiagGeneral) {   // one shape, every offset in range
        const int4 sh = __ldg(p.shapes + dc - 1);
        dr = __ldg(p.shape_dias + dc - 1);
        cb0 = sh.z - sh.x;
    }
    for (int rl = threadIdx.x; rl < nr; rl += kWinBlock) {
        const int r = row0 + rl;
        float acc = 0.f;
        if (SIGNED) {
            if (dc == kDiagGeneral) {
                acc = win_diag_general(p, xv, r);
            } else if (dc != kDiagNone) {
                for (int d = dr.x; d < dr.y; ++d) acc += xv(r + cb0 + __ldg(p.offsets + d));
            }
        }
        const int b = rp[rl] - t.nz0, e = rp[rl + 1] - t.nz0;
        for (int j = b; j < e; ++j) {
            const int w = cw[j];
            float v = xv(SIGNED ? (w >> 1) : w);
            if (SIGNED && !(w & 1)) v = -v;
            acc += v;
        }
        y[r] = acc;
    }
}

template <bool SIGNED>
__global__ void __launch_bounds__(kWinBlock, 1)
    spmv_window_kernel(DevPlan p, const float *__restrict__ x, float *__restrict__ y, int xa)
{
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem);
    int *const stages = reinterpret_cast<int *>(smem + 128);
    const int S = p.w_stages;
    const int stride = p.w_rp + p.w_cw + p.w_xw;            // ints per stage
    const int G = gridDim.x, nt = p.nwtiles;
    allow_next_grid();
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) mbar_init(bar + s, 2);  // index copies + x copy
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int s = 0; s < S; ++s) {
            const int t = blockIdx.x + s * G;
            if (t < nt) win_issue_index(p, p.wtiles[t], stages + s * stride, bar + s);
        }
    wait_prior_grid(x, y);
    if (threadIdx.x == 0) {
        asm volatile("fence.proxy.async.global;" ::: "memory");   // x written by earlier grids
        for (int s = 0; s < S; ++s) {
            const int t = blockIdx.x + s * G;
            if (t < nt) win_issue_x(p, p.wtiles[t], stages + s * stride, bar + s, x, xa != 0);
        }
    }
    int i = 0;
    for (int t = blockIdx.x; t < nt; t += G, ++i) {
        const int s = i % S;
        int *const st = stages + s * stride;
        const bool ok = mbar_wait(bar + s, (unsigned)(i / S) & 1u);
        if (!__syncthreads_and(ok)) {                       // every thread takes this branch
            if (threadIdx.x == 0) {
                atomicExch(p.err, 1);
                for (int j = i; j < i + S; ++j)               // copies still in flight land
                    if (blockIdx.x + j * G < nt) mbar_wait(bar + j % S, (unsigned)(j / S) & 1u);
            }
            return;
        }
        win_tile<SIGNED>(p, p.wtiles[t], st, x, y, xa != 0);
        __syncthreads();                                    // stage s is free again
        if (threadIdx.x == 0) {
            const int t2 = t + S * G;
            if (t2 < nt) {
                fence_async_shared();
                const Tile tt = p.wtiles[t2];
                win_issue_index(p, tt, st, bar + s);
                win_issue_x(p, tt, st, bar + s, x, xa != 0);
            }
        }
    }
}

int g_sms = 0;
int sms()
{
    if (g_sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
        if (g_sms <= 0) g_sms = 148;
    }
    return g_sms;
}

}  // namespace

size_t window_smem_bytes(const DevPlan &dp)
{
    return 128 + 4 * (size_t)dp.w_stages * (size_t)(dp.w_rp + dp.w_cw + dp.w_xw);
}

tc_status window_prepare(DevPlan &dp)
{
    if (dp.nwtiles <= 0) return TC_OK;
    const size_t smem = window_smem_bytes(dp);
    TC_CHECK(ensure_smem((const void *)spmv_window_kernel<false>, smem));
    TC_CHECK(ensure_smem((const void *)spmv_window_kernel<true>, smem));
    return TC_OK;
}

tc_status launch_window(const DevPlan &dp, const float *x, float *y, cudaStream_t s)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(dp.w_grid);
    cfg.blockDim = dim3(kWinBlock);
    cfg.dynamicSmemBytes = window_smem_bytes(dp);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = dp.pdl ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const int xa = (reinterpret_cast<uintptr_t>(x) & 15) == 0;
    if (dp.hybrid) TC_CUDA(cudaLaunchKernelEx(&cfg, spmv_window_kernel<true>, dp, x, y, xa));
    else TC_CUDA(cudaLaunchKernelEx(&cfg, spmv_window_kernel<false>, dp, x, y, xa));
    return TC_OK;
}

// ------------------------------------------------------------------ planner
// Window offsets [wlo, whi] of a plan: the shortest range of column - row
// that holds at least kWinCover of the matrix's accesses within +-kWinHalo
// (dense-diagonal terms and CSR words, rows sampled evenly when the matrix is
// large).  Built only on request (TC_FLAG_WINDOW).
bool plan_window(const tc_plan *p, const int *rp, const int *cw, std::vector<Tile> &wt, int *wlo, int *whi,
                 int *max_rows, int *max_nnz)
{
    wt.clear();
    const int M = p->M;
    const int flags = p->params.flags;
    const bool force = (flags & TC_FLAG_WINDOW) != 0;
    if (p->params.tile_mode != 2 || (flags & TC_FLAG_NO_WINDOW) || M == 0) return false;
    // Only on request (the flag, or the tuner when it times the window plan
    // faster): on the 9-point mesh (2048^2) the window kernel measured 108 us
    // per multiply against 52 us for the stream tiles, whose CTA-per-tile
    // grid keeps more loads in flight than one pipelined CTA per SM.
    if (!force) return false;
    const int H = kWinHalo;
    std::vector<int64_t> hist(2 * H + 1, 0);
    int64_t total = 0;
    const int step = std::max(1, M / (1 << 17));
    int64_t rows_seen = 0;
    for (int r = 0; r < M; r += step) {
        ++rows_seen;
        for (int j = rp[r]; j < rp[r + 1]; ++j) {
            const long c = p->hybrid ? (cw[j] >> 1) : cw[j];
            const long d = c - r;
            ++total;
            if (d >= -H && d <= H) ++hist[d + H];
        }
        if (r < p->row_start || r >= p->row_stop) continue;
        for (int s = 0; s < p->dia_shapes; ++s) {
            if (r < p->h_xStart[s] || r >= p->h_xStop[s]) continue;
            const int msub = p->h_xStop[s] - p->h_xStart[s];
            for (int n = p->h_nDiasPtr[s]; n < p->h_nDiasPtr[s + 1]; ++n) {
                const long cl = (long)r - p->h_xStart[s] + p->h_offsets[n];   // column inside the shape
                if (cl < 0 || cl >= msub) continue;
                const long d = p->h_yStart[s] + cl - r;
                ++total;
                if (d >= -H && d <= H) ++hist[d + H];
            }
        }
    }
    if (total == 0 || rows_seen == 0) return false;
    int64_t in = 0;
    for (int64_t v : hist) in += v;
    if (in == 0) return false;
    const int64_t target = std::max<int64_t>(1, (int64_t)(kWinCover * (double)in + 0.5));
    int best_lo = 0, best_hi = 2 * H;
    int64_t sum = 0;
    for (int lo = 0, hi = -1; lo <= 2 * H; ++lo) {   // shortest [lo, hi] with sum >= target
        while (sum < target && hi < 2 * H) sum += hist[++hi];
        if (sum < target) break;
        if (hi - lo < best_hi - best_lo) {
            best_lo = lo;
            best_hi = hi;
        }
        sum -= hist[lo];
    }
    *wlo = best_lo - H;
    *whi = best_hi - H;
    const int rows_cap = std::max(1, std::min(p->params.tile_rows, kWinRows));
    *max_rows = *max_nnz = 0;
    for (int r = 0; r < M;) {
        int n = 0;
        while (r + n < M && n < rows_cap && rp[r + n + 1] - rp[r] <= kWinNnz) ++n;
        if (n == 0) {                       // a row longer than a stage holds
            wt.clear();
            return false;
        }
        wt.push_back(Tile{r, rp[r], rp[r + n] - rp[r], tile_word(n, TILE_WINDOW)});
        *max_rows = std::max(*max_rows, n);
        *max_nnz = std::max(*max_nnz, rp[r + n] - rp[r]);
        r += n;
    }
    return true;
}

}  // namespace tc
