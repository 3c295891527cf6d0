// tc_tile.cuh -- device code of one multiply tile, shared by every multiply
// kernel (single plan, batch, served) so that a matrix gets bit-identical y
// whichever kernel runs it.
//
// A tile is a run of rows.  Its kind, chosen by the host planner from the
// tile's row lengths, fixes how many lanes share a row (1, 2, 4, ..., 32); a
// row longer than the planner's limit gets a whole CTA (TILE_LONG).  A lane
// group handles kRPT rows per pass and keeps their loads in flight together.
// Per row (FP32), each lane accumulates: the dense-diagonal terms of the
// offsets it owns (offset order), then its CSR entries in stored order (holes
// subtract, leftovers add); a butterfly reduction over the row's lanes ends
// it.  These are the terms of TaiChi.cu:1007-1040 in a fixed order.
//
// The row pointers and CSR words of a tile come either straight from global
// memory (GlobalSrc) or from a shared-memory copy that the TMA pipeline of the
// multiply kernel brought in ahead of time (SharedSrc); the arithmetic is the
// same for both.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "tc_internal.h"

namespace tc {

constexpr int kRPT = 4;   // rows per lane group per pass

__host__ __device__ inline int tile_rows_for(int lanes) { return (kBlock / lanes) * kRPT; }

template <bool SIGNED>
__device__ __forceinline__ float gather(const float *__restrict__ x, int c)
{
    if (SIGNED) {
        const float v = __ldg(x + (c >> 1));
        return (c & 1) ? v : -v;
    }
    return __ldg(x + c);
}

// Programmatic dependent launch: a kernel reads only immutable plan data
// before wait_prior_grid(); x is read and y written after it, when every grid
// earlier in the stream has finished and its writes are visible.
__device__ __forceinline__ void wait_prior_grid() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void allow_next_grid() { asm volatile("griddepcontrol.launch_dependents;" :::); }

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Tile-relative row pointers / CSR words read from global memory.
struct GlobalSrc {
    const int *rp;     // &rowptr[row0]
    const int *cw;     // &cols[nz0]
    int nz0;
    __device__ __forceinline__ int row(int r) const { return __ldg(rp + r) - nz0; }
    __device__ __forceinline__ int word(int j) const { return __ldg(cw + j); }
};

// The same read from a shared-memory copy (aligned-down starts: rp_off / cw_off).
struct SharedSrc {
    const int *rp;
    const int *cw;
    int nz0;
    __device__ __forceinline__ int row(int r) const { return rp[r] - nz0; }
    __device__ __forceinline__ int word(int j) const { return cw[j]; }
};

// Adds the dense-diagonal terms of rows row0 + base + k*G + g (k < kRPT) to
// acc[k]; the shape's offsets are split over the row's lanes.  Offset `off`
// of a shape covers rows [xStart + max(0,-off), xStop - max(0,off)).
template <int LANES>
__device__ __forceinline__ void diag_terms(const DevPlan &p, const float *__restrict__ x, int row0,
                                           int nr, int base, int g, int lane, float (&acc)[kRPT])
{
    constexpr int G = kBlock / LANES;
    const int lo = row0 + base, hi = row0 + min(nr, base + G * kRPT);   // rows of this pass
    if (hi <= p.row_start || lo >= p.row_stop) return;
    for (int s = 0; s < p.dia_shapes; ++s) {
        const int4 sh = __ldg(p.shapes + s);          // xStart, xStop, yStart, Msub
        if (hi <= sh.x || lo >= sh.y) continue;       // uniform across the CTA
        const int2 dr = __ldg(p.shape_dias + s);
        const int cb = sh.z - sh.x;                   // column = row + cb + off
        for (int n = dr.x + lane; n < dr.y; n += LANES) {
            const int off = __ldg(p.offsets + n);
            const int a = sh.x + max(0, -off), b = sh.y - max(0, off);
            float v[kRPT];
#pragma unroll
            for (int k = 0; k < kRPT; ++k) {
                const int rl = base + k * G + g, r = row0 + rl;
                v[k] = (rl < nr && r >= a && r < b) ? __ldg(x + r + cb + off) : 0.f;
            }
#pragma unroll
            for (int k = 0; k < kRPT; ++k) acc[k] += v[k];
        }
    }
}

// One pass (kRPT rows per lane group) of a TILE_L<LANES> tile.
template <bool SIGNED, int LANES, class Src>
__device__ __forceinline__ void rows_pass(const DevPlan &p, int row0, int nr, int base,
                                          const Src &src, const float *__restrict__ x,
                                          float *__restrict__ y, bool wait)
{
    constexpr int G = kBlock / LANES;
    const int g = threadIdx.x / LANES;
    const int lane = threadIdx.x & (LANES - 1);
    int rb[kRPT], re[kRPT];
#pragma unroll
    for (int k = 0; k < kRPT; ++k) {
        const int r = base + k * G + g;
        const bool ok = r < nr;
        rb[k] = ok ? src.row(r) : 0;
        re[k] = ok ? src.row(r + 1) : 0;
    }
    // first round of CSR words: immutable plan data, loaded before the wait
    int c[kRPT];
#pragma unroll
    for (int k = 0; k < kRPT; ++k) {
        const int j = rb[k] + lane;
        c[k] = j < re[k] ? src.word(j) : -1;
    }
    if (wait) wait_prior_grid();
    float acc[kRPT];
#pragma unroll
    for (int k = 0; k < kRPT; ++k) acc[k] = 0.f;
    if (p.dia_shapes > 0) diag_terms<LANES>(p, x, row0, nr, base, g, lane, acc);
    for (int j0 = lane;;) {
        float v[kRPT];
#pragma unroll
        for (int k = 0; k < kRPT; ++k) v[k] = c[k] >= 0 ? gather<SIGNED>(x, c[k]) : 0.f;
#pragma unroll
        for (int k = 0; k < kRPT; ++k)
            if (c[k] >= 0) acc[k] += v[k];
        j0 += LANES;
        bool more = false;
#pragma unroll
        for (int k = 0; k < kRPT; ++k) {
            const int j = rb[k] + j0;
            const bool ok = j < re[k];
            c[k] = ok ? src.word(j) : -1;
            more |= ok;
        }
        if (!__any_sync(0xffffffffu, more)) break;
    }
#pragma unroll
    for (int k = 0; k < kRPT; ++k) {
#pragma unroll
        for (int o = LANES / 2; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
        const int r = base + k * G + g;
        if (lane == 0 && r < nr) y[row0 + r] = acc[k];
    }
}

template <bool SIGNED, int LANES, class Src>
__device__ __forceinline__ void tile_rows(const DevPlan &p, const Tile &t, const Src &src,
                                          const float *__restrict__ x, float *__restrict__ y,
                                          bool wait)
{
    constexpr int G = kBlock / LANES;
    const int nr = tile_nrows(t);
    for (int base = 0; base < nr; base += G * kRPT)
        rows_pass<SIGNED, LANES>(p, t.row0, nr, base, src, x, y, wait);
}

// One lane per row: a thread owns up to kRPT consecutive rows and walks
// their CSR words straight through (no lock-step rounds), after adding each
// row's dense-diagonal terms.  Same per-row order as rows_pass.
template <bool SIGNED, class Src>
__device__ __forceinline__ void tile_rows1(const DevPlan &p, const Tile &t, const Src &src,
                                           const float *__restrict__ x, float *__restrict__ y,
                                           bool wait)
{
    const int nr = tile_nrows(t), row0 = t.row0;
    for (int base = 0; base < nr; base += kBlock * kRPT) {
        const int n = min(nr - base, kBlock * kRPT);
        const int q = (n + kBlock - 1) / kBlock;            // rows per thread, 1..kRPT
        const int lo = base + (int)threadIdx.x * q;
        const int hi = min(lo + q, base + n);               // this thread's rows [lo, hi)
        int e[kRPT + 1];
#pragma unroll
        for (int k = 0; k <= kRPT; ++k) e[k] = lo < hi ? src.row(min(lo + k, hi)) : 0;
        if (wait) wait_prior_grid();
        float acc[kRPT];
#pragma unroll
        for (int k = 0; k < kRPT; ++k) acc[k] = 0.f;
        if (p.dia_shapes > 0 && lo < hi && row0 + hi > p.row_start && row0 + lo < p.row_stop) {
            for (int s = 0; s < p.dia_shapes; ++s) {
                const int4 sh = __ldg(p.shapes + s);        // xStart, xStop, yStart, Msub
                if (row0 + hi <= sh.x || row0 + lo >= sh.y) continue;
                const int2 dr = __ldg(p.shape_dias + s);
                const int cb = sh.z - sh.x;
                for (int d = dr.x; d < dr.y; ++d) {
                    const int off = __ldg(p.offsets + d);
                    const int a = sh.x + max(0, -off), b = sh.y - max(0, off);
                    float v[kRPT];
#pragma unroll
                    for (int k = 0; k < kRPT; ++k) {
                        const int r = row0 + lo + k;
                        v[k] = (lo + k < hi && r >= a && r < b) ? __ldg(x + r + cb + off) : 0.f;
                    }
#pragma unroll
                    for (int k = 0; k < kRPT; ++k) acc[k] += v[k];
                }
            }
        }
#pragma unroll
        for (int k = 0; k < kRPT; ++k) {
#pragma unroll 4
            for (int j = e[k]; j < e[k + 1]; ++j) acc[k] += gather<SIGNED>(x, src.word(j));
        }
#pragma unroll
        for (int k = 0; k < kRPT; ++k)
            if (lo + k < hi) y[row0 + lo + k] = acc[k];
    }
}

// One row with more entries than the planner's per-tile limit: the whole CTA
// strides over it; warp sums are combined in warp order.
template <bool SIGNED>
__device__ void long_row(const DevPlan &p, const Tile &t, const float *__restrict__ x,
                         float *__restrict__ y, bool wait)
{
    __shared__ float red[kBlock / 32];
    constexpr int U = 8;
    const int tid = threadIdx.x;
    const int *__restrict__ cols = p.cols + t.nz0;
    float acc = 0.f;
    bool waited = !wait;
    // dense-diagonal terms of the row first (thread-strided offsets)
    if (!waited) { wait_prior_grid(); waited = true; }
    const int r = t.row0;
    if (p.dia_shapes > 0 && r >= p.row_start && r < p.row_stop)
        for (int s = 0; s < p.dia_shapes; ++s) {
            const int4 sh = __ldg(p.shapes + s);
            if (r < sh.x || r >= sh.y) continue;
            const int2 dr = __ldg(p.shape_dias + s);
            for (int n = dr.x + tid; n < dr.y; n += kBlock) {
                const int c = r - sh.x + sh.z + __ldg(p.offsets + n);
                if (c >= sh.z && c < sh.z + sh.w) acc += __ldg(x + c);
            }
        }
    for (int base = 0; base < t.nnz; base += kBlock * U) {
        int c[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = base + u * kBlock + tid;
            c[u] = i < t.nnz ? __ldg(cols + i) : -1;
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (c[u] >= 0) acc += gather<SIGNED>(x, c[u]);
    }
    acc = warp_sum(acc);
    if ((tid & 31) == 0) red[tid >> 5] = acc;
    __syncthreads();
    if (tid < 32) {
        float v = tid < kBlock / 32 ? red[tid] : 0.f;
        v = warp_sum(v);
        if (tid == 0) y[r] = v;
    }
    __syncthreads();
}

template <bool SIGNED, class Src>
__device__ __forceinline__ void run_tile_src(const DevPlan &p, const Tile &t, const Src &src,
                                             const float *__restrict__ x, float *__restrict__ y,
                                             bool wait)
{
    switch (tile_kind(t)) {
    case TILE_L1: tile_rows1<SIGNED>(p, t, src, x, y, wait); break;
    case TILE_L2: tile_rows<SIGNED, 2>(p, t, src, x, y, wait); break;
    case TILE_L4: tile_rows<SIGNED, 4>(p, t, src, x, y, wait); break;
    case TILE_L8: tile_rows<SIGNED, 8>(p, t, src, x, y, wait); break;
    case TILE_L16: tile_rows<SIGNED, 16>(p, t, src, x, y, wait); break;
    case TILE_L32: tile_rows<SIGNED, 32>(p, t, src, x, y, wait); break;
    default: long_row<SIGNED>(p, t, x, y, wait); break;
    }
}

// A tile read straight from global memory.
template <bool SIGNED>
__device__ __forceinline__ void run_tile(const DevPlan &p, const Tile &t, const float *__restrict__ x,
                                         float *__restrict__ y, bool wait = true)
{
    const GlobalSrc src{p.rowptr + t.row0, p.cols + t.nz0, t.nz0};
    run_tile_src<SIGNED>(p, t, src, x, y, wait);
}

}  // namespace tc
