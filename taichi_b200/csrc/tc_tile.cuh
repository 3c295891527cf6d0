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

// A load of x: a coherent global load (ld.global, cached in L1 and L2), never
// the read-only path.  Under programmatic dependent launch a multiply is
// resident while the grid before it may still be writing its x, so x is not
// read-only for the kernel's lifetime -- the contract of ld.global.nc, whose
// loads may be scheduled ahead of griddepcontrol.wait.  (With __ldg here,
// chained multiplies v <- A v read stale x in up to 6 % of the rows.)
// Plan arrays (row pointers, CSR words, shapes, offsets) never change while
// a plan exists and keep __ldg.
__device__ __forceinline__ float ldx(const float *p)
{
    float v;
    asm("ld.global.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}

template <bool SIGNED>
__device__ __forceinline__ float gather(const float *__restrict__ x, int c)
{
    if (SIGNED) {
        const float v = ldx(x + (c >> 1));
        return (c & 1) ? v : -v;
    }
    return ldx(x + c);
}

// gather() of a signed word known to be an addition (c & 1 set: a plan
// with no holes in its dense diagonals), without the sign select.
template <bool SIGNED, bool POS>
__device__ __forceinline__ float gather_pos(const float *__restrict__ x, int c)
{
    if (SIGNED && POS) return ldx(x + (c >> 1));
    return gather<SIGNED>(x, c);
}

// Programmatic dependent launch: a kernel reads only immutable plan data
// before wait_prior_grid(); x is read and y written after it, when every grid
// earlier in the stream has finished and its writes are visible.
__device__ __forceinline__ void wait_prior_grid() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void allow_next_grid() { asm volatile("griddepcontrol.launch_dependents;" :::); }

// The wait, with the vector pointers passed through the same asm statement:
// every load of x and store of y made through them afterwards depends on the
// wait in the compiler's view too.  A memory clobber alone does not order
// them -- x and y are __restrict__, so the compiler may take the asm for
// unable to touch them and move x loads ahead of it, where they would race
// an earlier grid's writes of x.  The loads themselves are ldx() (coherent),
// which the assembler keeps behind griddepcontrol.wait.
__device__ __forceinline__ void wait_prior_grid(const float *__restrict__ &x, float *__restrict__ &y)
{
    asm volatile("griddepcontrol.wait;" : "+l"(x), "+l"(y)::"memory");
}

// The same dependence for a thread that waited earlier (the later tiles of a
// persistent CTA): x and y re-derived after everything the thread did so far.
__device__ __forceinline__ void after_wait(const float *__restrict__ &x, float *__restrict__ &y)
{
    asm volatile("" : "+l"(x), "+l"(y)::"memory");
}

// Starts one bulk read of x[r0, r0 + n) into L2 (the whole 16-byte granules
// inside x[0, N) only; nothing is prefetched from outside the vector).  A
// tile's gathers land mostly near its own rows, and most of the window is
// read by some gather: streaming the window in at the tile's start, while
// its row pointers and words are still in flight, turns scattered x misses
// into L2 hits (R-MAT scale 20: 5.9 -> 5.5 µs per multiply, with the wide
// kernel no longer waiting for its tile record first).  An L2 prefetch
// is only a hint and L2 is where every SM's writes land, so it may be issued
// before wait_prior_grid(): a later write of x by an earlier grid still
// reaches the loads that follow the wait.
__device__ __forceinline__ void prefetch_x_window(const float *x, int N, int r0, int n)
{
    const int a = max(r0, 0), b = min(r0 + n, N);
    if (b <= a) return;
    const uintptr_t lo = (reinterpret_cast<uintptr_t>(x + a) + 15) & ~uintptr_t(15);
    const uintptr_t hi = reinterpret_cast<uintptr_t>(x + b) & ~uintptr_t(15);
    if (hi > lo)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(lo), "r"((unsigned)(hi - lo)) : "memory");
}

// One bulk L2 prefetch of [p, p + bytes): p 16-byte aligned, bytes a multiple
// of 16, the whole range inside one allocation.
__device__ __forceinline__ void prefetch_l2(const void *p, unsigned bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// L2 prefetch of a[i0, i1) of a plan array (row pointers or CSR words),
// rounded out to 16 bytes: the plan's arrays start 256-byte aligned and are
// padded by 16 bytes past their last element, so the rounded span stays
// inside the allocation.
__device__ __forceinline__ void prefetch_span(const int *a, int i0, int i1)
{
    const uintptr_t lo = reinterpret_cast<uintptr_t>(a + i0) & ~uintptr_t(15);
    const uintptr_t hi = (reinterpret_cast<uintptr_t>(a + i1) + 15) & ~uintptr_t(15);
    if (hi > lo) prefetch_l2(reinterpret_cast<const void *>(lo), (unsigned)(hi - lo));
}

// Row pointers and CSR words of rows [r0, r1), whose words are [z0, z1),
// brought into L2 about a wave before the CTA that reads them starts: the
// CTA's row-pointer and word loads then hit L2 instead of waiting on HBM,
// and the HBM reads run ahead of the dependent load chains.  Immutable plan
// data, so it may be issued at any time.
__device__ __forceinline__ void prefetch_rows_ahead(const DevPlan &p, int r0, int r1, int z0, int z1)
{
    prefetch_span(p.rowptr, r0, r1 + 1);
    prefetch_span(p.cols, z0, z1);
}

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
                v[k] = (rl < nr && r >= a && r < b) ? ldx(x + r + cb + off) : 0.f;
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
    if (wait) wait_prior_grid(x, y);
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

// Dense-diagonal terms of one row, offsets in order.
__device__ __forceinline__ float diag_row(const DevPlan &p, const float *__restrict__ x, int r);

// One lane per row, rows strided over the CTA (coalesced y and diagonal
// loads): per row the diagonal terms in offset order, then the CSR words in
// stored order -- the order of rows_pass<LANES = 1>.
template <bool SIGNED, class Src>
__device__ __forceinline__ void tile_rows_seq(const DevPlan &p, const Tile &t, const Src &src,
                                              const float *__restrict__ x, float *__restrict__ y,
                                              bool wait)
{
    const int nr = tile_nrows(t), row0 = t.row0;
    if (wait) wait_prior_grid(x, y);
    for (int rl = threadIdx.x; rl < nr; rl += kBlock) {
        const int b = src.row(rl), e = src.row(rl + 1);
        float acc = p.dia_shapes > 0 ? diag_row(p, x, row0 + rl) : 0.f;
#pragma unroll 2
        for (int j = b; j < e; ++j) acc += gather<SIGNED>(x, src.word(j));
        y[row0 + rl] = acc;
    }
}

// ---------------------------------------------------------------- merge tile
// Load-balanced walk of a tile (the merge-path split of Merrill & Garland):
// the tile's nr row ends and nz CSR entries form one sequence of nr + nz
// items, cut into equal runs of L = ceil((nr + nz) / kBlock) items, one run
// per thread.  A thread finds where its run starts by a binary search on the
// row pointers, gathers x for its run's entries eight at a time, and closes
// the rows that end inside its run.  A row that starts in an earlier run
// leaves a carry there; the thread that closes the row adds the carries of
// the runs before it in thread order, so the sum order is fixed by the tile
// alone.  Then each row gets its dense-diagonal terms and y is stored once.
constexpr int kMergeRows = 2048;          // most rows in one merge tile
constexpr int kMergeBatch = 8;            // gathers in flight per thread

// Largest i in [0, nr] whose first CSR entry plus i does not pass item d.
template <class Src>
__device__ __forceinline__ int merge_split(const Src &src, int nr, int nz, int d)
{
    int lo = max(0, d - nz), hi = min(d, nr);
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (src.row(mid) + mid <= d) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Dense-diagonal terms of one row, offsets in order, kDiagU offsets' loads
// issued before their adds (a wide band's terms do not wait on each other).
constexpr int kDiagU = 4;

__device__ __forceinline__ float diag_row(const DevPlan &p, const float *__restrict__ x, int r)
{
    float acc = 0.f;
    if (r < p.row_start || r >= p.row_stop) return acc;
    for (int s = 0; s < p.dia_shapes; ++s) {
        const int4 sh = __ldg(p.shapes + s);
        if (r < sh.x || r >= sh.y) continue;
        const int2 dr = __ldg(p.shape_dias + s);
        const int cb = r - sh.x + sh.z;
        for (int d = dr.x; d < dr.y; d += kDiagU) {
            float v[kDiagU];
            bool in[kDiagU];
#pragma unroll
            for (int k = 0; k < kDiagU; ++k) {
                const int c = d + k < dr.y ? cb + __ldg(p.offsets + d + k) : -1;
                in[k] = c >= sh.z && c < sh.z + sh.w;
                v[k] = in[k] ? ldx(x + c) : 0.f;
            }
#pragma unroll
            for (int k = 0; k < kDiagU; ++k)
                if (in[k]) acc += v[k];
        }
    }
    return acc;
}

// Shared memory of the merge and stream tiles: one union per kernel, used by
// every instantiation of the tile code in that kernel.
struct MergeSmem {
    float rsum[kMergeRows];
    float carry[kBlock];
    int crow[kBlock];
};
union TileSmem {
    MergeSmem merge;
    float4 vals4[(kStreamNnz + 8 + (kStreamNnz + 8) / 32 + 4) / 4];   // alignment of the stream slots
    float vals[kStreamNnz + 8 + (kStreamNnz + 8) / 32 + 1];   // stream tiles (see vslot)
};
__device__ __forceinline__ TileSmem &tile_smem()
{
    __shared__ TileSmem s;
    return s;
}

template <bool SIGNED, class Src>
__device__ void tile_merge(const DevPlan &p, const Tile &t, const Src &src,
                           const float *__restrict__ x, float *__restrict__ y, bool wait)
{
    float *const rsum = tile_smem().merge.rsum;
    float *const carry = tile_smem().merge.carry;
    int *const crow = tile_smem().merge.crow;
    const int nr = tile_nrows(t), nz = t.nnz, row0 = t.row0, tid = threadIdx.x;
    const int total = nr + nz;
    const int L = (total + kBlock - 1) / kBlock;
    const int d0 = min(tid * L, total), d1 = min(d0 + L, total);
    const int i0 = merge_split(src, nr, nz, d0);
    int i1 = __shfl_down_sync(0xffffffffu, i0, 1);       // the next run starts where this ends
    if ((tid & 31) == 31) i1 = merge_split(src, nr, nz, d1);
    const int j0 = d0 - i0, j1 = d1 - i1;
    if (wait) wait_prior_grid(x, y);
    float acc = 0.f;
    int r = i0;
    int rend = r < nr ? src.row(r + 1) : nz;
    for (int jb = j0; jb < j1; jb += kMergeBatch) {
        float v[kMergeBatch];
#pragma unroll
        for (int u = 0; u < kMergeBatch; ++u) {
            const int j = jb + u;
            v[u] = j < j1 ? gather<SIGNED>(x, src.word(j)) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < kMergeBatch; ++u) {
            const int j = jb + u;
            if (j < j1) {
                while (j >= rend) {               // rows that end before entry j
                    rsum[r] = acc;
                    acc = 0.f;
                    ++r;
                    rend = src.row(r + 1);
                }
                acc += v[u];
            }
        }
    }
    while (r < i1) {                              // rows ending at the end of the run
        rsum[r] = acc;
        acc = 0.f;
        ++r;
    }
    const bool partial = r < nr && j1 > max(j0, r < nr ? src.row(r) : nz);
    crow[tid] = partial ? r : -1;
    carry[tid] = acc;
    __syncthreads();
    if (i1 > i0 && tid > 0 && crow[tid - 1] == i0) {   // row i0 began in earlier runs
        float add = 0.f;
        for (int u = tid - 1; u >= 0 && crow[u] == i0; --u) add += carry[u];
        rsum[i0] += add;
    }
    __syncthreads();
    for (int rr = tid; rr < nr; rr += kBlock) {
        float v = rsum[rr];
        if (p.dia_shapes > 0) v += diag_row(p, x, row0 + rr);
        y[row0 + rr] = v;
    }
    __syncthreads();                              // rsum / carry are reused by the next tile
}

// ---------------------------------------------------------------- stream tile
// Entry-parallel gather, row-parallel sum.  The tile's CSR words are read as
// the 16-byte aligned int4s that cover them, coalesced across the CTA (the
// cols array is 256-byte aligned and zero-padded past its end, so the window
// never leaves it); each thread turns its kStreamQ int4s per round into
// kStreamQ * 4 signed x terms, all loads in flight together, and stores them
// as float4s in shared memory at their window position (entry j of the tile
// at slot vslot(lead + j)).  Words of the window outside the tile are valid column
// words of neighbouring tiles (or the zero padding, column 0), so their
// gathers stay inside x and their slots are never read.  Then each row's
// dense-diagonal terms (offset order) and entries (stored order) are added
// by one thread: the order of tile_rows_seq, so a matrix gets the same y from
// every one-lane tile kind.  TILE_STREAM strides single rows over the CTA;
// TILE_STREAM4 gives each thread runs of 4 consecutive rows (int4
// row-pointer loads, float4 y stores) for tiles of many short rows.  The
// first round's CSR words and the row pointers are immutable plan data, read
// before wait_prior_grid().
constexpr int kStreamQ = 2;   // int4 CSR words per thread per round

struct StreamWords {
    const int4 *cq;   // aligned-down start of the tile's CSR words
    int lead;         // words before nz0 in the first int4
    int nq;           // int4s covering the tile
    int4 w[kStreamQ]; // this thread's first-round words
};

__device__ __forceinline__ void stream_words_first(const DevPlan &p, const Tile &t, StreamWords &sw)
{
    sw.lead = t.nz0 & 3;
    sw.cq = reinterpret_cast<const int4 *>(p.cols + (t.nz0 - sw.lead));
    sw.nq = (sw.lead + t.nnz + 3) >> 2;
#pragma unroll
    for (int q = 0; q < kStreamQ; ++q) {
        const int i = threadIdx.x + q * kBlock;
        sw.w[q] = i < sw.nq ? __ldg(sw.cq + i) : make_int4(0, 0, 0, 0);
    }
}

// Shared-memory slot of window entry j of a stream tile of a plan whose
// rows mostly have a length that is a multiple of 8 (DevPlan::skew): one
// spare slot per 32 entries, so threads summing rows of equal length L read
// banks that differ (without the skew, rows of exactly 32 entries put every
// lane of a warp on one bank: a banded matrix of such rows ran 341 us per
// multiply against 99 us with it).  Other plans keep slot j (float4 stores,
// no index arithmetic: the skew cost the 9-point mesh 4 %).
__device__ __forceinline__ int vslot(int j) { return j + (j >> 5); }

// vals[slot(lead + j)] = signed x term of entry j of the tile; ends with a
// barrier.
template <bool SIGNED>
__device__ __forceinline__ void stream_gather(const float *__restrict__ x, float *vals, StreamWords &sw, bool skew)
{
    const int tid = threadIdx.x;
    for (int base = 0; base < sw.nq; base += kStreamQ * kBlock) {
        if (base > 0) {
#pragma unroll
            for (int q = 0; q < kStreamQ; ++q) {
                const int i = base + tid + q * kBlock;
                sw.w[q] = i < sw.nq ? __ldg(sw.cq + i) : make_int4(0, 0, 0, 0);
            }
        }
        // signed words: every slot is gathered -- a slot past the window
        // holds word 0, a load of x[0] that is never stored -- so no branch
        // surrounds the loads (mesh, stream tiles: 48.1 -> 45.7 us); plain
        // words keep the branch (the unconditional form spills in the
        // plain 8-CTA build)
        float4 v[kStreamQ];
#pragma unroll
        for (int q = 0; q < kStreamQ; ++q) {
            if (SIGNED || base + tid + q * kBlock < sw.nq) {
                v[q].x = gather<SIGNED>(x, sw.w[q].x);
                v[q].y = gather<SIGNED>(x, sw.w[q].y);
                v[q].z = gather<SIGNED>(x, sw.w[q].z);
                v[q].w = gather<SIGNED>(x, sw.w[q].w);
            }
        }
#pragma unroll
        for (int q = 0; q < kStreamQ; ++q) {
            const int i = base + tid + q * kBlock;
            if (i < sw.nq) {
                if (skew) {
                    float *d = vals + vslot(4 * i);  // 4i .. 4i + 3 share one 32-entry group
                    d[0] = v[q].x;
                    d[1] = v[q].y;
                    d[2] = v[q].z;
                    d[3] = v[q].w;
                } else {
                    reinterpret_cast<float4 *>(vals)[i] = v[q];
                }
            }
        }
    }
    __syncthreads();
}

// Dense-diagonal terms of row r of a tile of diagonal class dc: the terms
// and order of diag_row, without the per-row shape search when the class
// names the tile's one shape.
__device__ __forceinline__ float diag_tile_row(const DevPlan &p, const float *__restrict__ x, int dc, int r)
{
    if (dc == kDiagNone) return 0.f;
    if (dc == kDiagGeneral) return diag_row(p, x, r);
    if (p.dn > 0 && p.dn <= 4) {
        // the plan's one shape, every offset inside it for this tile's rows:
        // the columns' shifts come with the plan descriptor (no shape or
        // offset reads), offsets in order
        float v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = u < p.dn ? ldx(x + r + p.d_col[u]) : 0.f;
        float acc = 0.f;
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (u < p.dn) acc += v[u];
        return acc;
    }
    const int4 sh = __ldg(p.shapes + dc - 1);
    const int2 dr = __ldg(p.shape_dias + dc - 1);
    const float *__restrict__ xr = x + (r - sh.x + sh.z);
    float acc = 0.f;
    for (int d = dr.x; d < dr.y; d += kDiagU) {
        float v[kDiagU];
#pragma unroll
        for (int k = 0; k < kDiagU; ++k) v[k] = d + k < dr.y ? ldx(xr + __ldg(p.offsets + d + k)) : 0.f;
#pragma unroll
        for (int k = 0; k < kDiagU; ++k)
            if (d + k < dr.y) acc += v[k];
    }
    return acc;
}

template <bool SIGNED>
__device__ void tile_stream(const DevPlan &p, const Tile &t, const float *__restrict__ x,
                            float *__restrict__ y, bool wait)
{
    float *const vals = tile_smem().vals;
    constexpr int RQ = kStreamRows / kBlock;
    const int tid = threadIdx.x, nr = tile_nrows(t), row0 = t.row0, dc = tile_dclass(t);
    StreamWords sw;
    stream_words_first(p, t, sw);
    const int base = t.nz0 - sw.lead;                           // rowptr value of vals[0]
    int rb[RQ], re[RQ];
#pragma unroll
    for (int k = 0; k < RQ; ++k) {
        const int rl = tid + k * kBlock;
        const bool ok = rl < nr;
        rb[k] = ok ? __ldg(p.rowptr + row0 + rl) - base : 0;
        re[k] = ok ? __ldg(p.rowptr + row0 + rl + 1) - base : 0;
    }
    if (wait) wait_prior_grid(x, y);
    stream_gather<SIGNED>(x, vals, sw, p.skew);
    // (Loading the rows' diagonal terms while the gathers are in flight
    // measured slower on the mesh: into registers 69.5 against 65.6 us; as
    // the tile's x segment staged in shared memory 58.3 against 52.5 us.)
#pragma unroll
    for (int k = 0; k < RQ; ++k) {
        const int rl = tid + k * kBlock;
        if (rl < nr) {
            float acc = diag_tile_row(p, x, dc, row0 + rl);
            if (p.skew) {
                for (int j = rb[k]; j < re[k]; ++j) acc += vals[vslot(j)];
            } else {
                for (int j = rb[k]; j < re[k]; ++j) acc += vals[j];
            }
            y[row0 + rl] = acc;
        }
    }
    __syncthreads();                                            // vals is reused by the next tile
}

// TILE_STREAM4: row0 is a multiple of 4 (the row pointers' int4 loads are
// aligned; the array is padded by 16 bytes past rowptr[M], and rows past the
// tile are masked), at most kStream4Rows rows.
template <bool SIGNED>
__device__ void tile_stream4(const DevPlan &p, const Tile &t, const float *__restrict__ x,
                             float *__restrict__ y, bool wait)
{
    float *const vals = tile_smem().vals;
    constexpr int GQ = kStream4Rows / (4 * kBlock);             // row groups per thread
    const int tid = threadIdx.x, nr = tile_nrows(t), row0 = t.row0, dc = tile_dclass(t);
    StreamWords sw;
    stream_words_first(p, t, sw);
    const int base = t.nz0 - sw.lead;
    int4 rp[GQ];
    int rp4[GQ];
#pragma unroll
    for (int k = 0; k < GQ; ++k) {
        const int g = 4 * (tid + k * kBlock);                   // first row of the group
        const bool ok = g < nr;
        rp[k] = ok ? __ldg(reinterpret_cast<const int4 *>(p.rowptr + row0 + g)) : make_int4(0, 0, 0, 0);
        rp4[k] = ok ? __ldg(p.rowptr + row0 + min(g + 4, nr)) : 0;
    }
    if (wait) wait_prior_grid(x, y);
    stream_gather<SIGNED>(x, vals, sw, p.skew);
#pragma unroll
    for (int k = 0; k < GQ; ++k) {
        const int g = 4 * (tid + k * kBlock);
        if (g >= nr) continue;
        const int b[5] = {rp[k].x - base, rp[k].y - base, rp[k].z - base, rp[k].w - base, rp4[k] - base};
        float acc[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            acc[u] = 0.f;
            if (g + u < nr) {
                acc[u] = diag_tile_row(p, x, dc, row0 + g + u);
                const int e = g + u + 1 < nr ? b[u + 1] : b[4];
                if (p.skew) {
                    for (int j = b[u]; j < e; ++j) acc[u] += vals[vslot(j)];
                } else {
                    for (int j = b[u]; j < e; ++j) acc[u] += vals[j];
                }
            }
        }
        float *yr = y + row0 + g;
        if (g + 4 <= nr && (reinterpret_cast<uintptr_t>(yr) & 15) == 0) {
            *reinterpret_cast<float4 *>(yr) = make_float4(acc[0], acc[1], acc[2], acc[3]);
        } else {
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (g + u < nr) yr[u] = acc[u];
        }
    }
    __syncthreads();                                            // vals is reused by the next tile
}

// Adds to acc[u] the dense-diagonal terms of rows r + u, u < n <= 4, of a
// tile of diagonal class dc: the terms and order of diag_row.  For a
// one-shape class the shape is read once for the 4 rows and each offset's 4
// x loads go out together.
__device__ __forceinline__ void diag_run4(const DevPlan &p, const float *__restrict__ x, int dc, int r, int n,
                                          float (&acc)[4])
{
    if (dc == kDiagNone) return;
    if (dc == kDiagGeneral) {
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (u < n) acc[u] += diag_row(p, x, r + u);
        return;
    }
    const int4 sh = __ldg(p.shapes + dc - 1);
    const int2 dr = __ldg(p.shape_dias + dc - 1);
    const float *__restrict__ xr = x + (r - sh.x + sh.z);
#pragma unroll 2
    for (int d = dr.x; d < dr.y; ++d) {
        const int off = __ldg(p.offsets + d);
        float v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = u < n ? ldx(xr + u + off) : 0.f;
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (u < n) acc[u] += v[u];
    }
}

// Direct tiles: runs of 4 consecutive rows per thread, read straight from
// global memory with no shared memory and no barrier -- for tiles whose rows
// average at most one entry, where a thread's 4 rows hold a handful of
// consecutive CSR words.  Row pointers come as one int4 (row0 % 4 == 0) plus
// the run's end; the first kDirectW words of the run and their gathers are
// all in flight together, each word added to the row that owns it (words in
// stored order, after the row's dense-diagonal terms: the order of
// tile_rows_seq); a run with more words walks the rest one at a time.
// TILE_DIRECT4 tiles (up to 1024 rows) give each of a 256-thread CTA's
// threads one run; TILE_DIRECT_WIDE tiles (up to 4096 rows) are run by the
// 1024-thread direct kernel, one run per thread, or by a 256-thread CTA as
// four passes of runs (batch and served launches) -- the same rows, terms and
// order either way.  (Two runs per thread with all loads in flight measured
// slower on R-MAT; four run out of registers.)
constexpr int kDirectW = 4;
// The whole-run path (direct_run_full) keeps more words of a run in flight:
// a run's words past the first W are walked one at a time, each a word load
// then a gather, and on R-MAT scale 20 a run of 4 rows holds more than 4
// words in 10 % of the runs -- 97 % of the warps -- more than 6 in 1.2 %
// (32 % of the warps), more than 8 in 0.08 %.  Measured per multiply
// (K = 2,000, one box): plain words W = 4 / 6 / 8: 4.74 / 4.52 / 4.71 µs;
// signed words (self-loop plan) 5.29 / 5.30 / 5.20 µs.
template <bool SIGNED>
constexpr int direct_w_full() { return SIGNED ? 8 : 6; }

// The run of rows [row0 + g, row0 + g + 4) of a direct tile of nr rows from
// row0 and diagonal class dc, g a multiple of 4.
template <bool SIGNED>
__device__ __forceinline__ void direct_run(const DevPlan &p, int row0, int nr, int dc, const float *__restrict__ x,
                                           float *__restrict__ y, bool wait, int g)
{
    if (g >= nr) {
        if (wait) wait_prior_grid(x, y);
        return;
    }
    const int4 r4 = __ldg(reinterpret_cast<const int4 *>(p.rowptr + row0 + g));
    const int e4 = __ldg(p.rowptr + row0 + min(g + 4, nr));
    // row u of the run holds words [b[u], b[u+1]); rows past the tile hold none
    const int b[5] = {r4.x, g + 1 < nr ? r4.y : e4, g + 2 < nr ? r4.z : e4, g + 3 < nr ? r4.w : e4, e4};
    int c[kDirectW];
#pragma unroll
    for (int w = 0; w < kDirectW; ++w) c[w] = b[0] + w < e4 ? __ldg(p.cols + b[0] + w) : 0;
    if (wait) wait_prior_grid(x, y);
    float v[kDirectW];
#pragma unroll
    for (int w = 0; w < kDirectW; ++w) v[w] = b[0] + w < e4 ? gather<SIGNED>(x, c[w]) : 0.f;
    float acc[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) acc[u] = 0.f;
    if (SIGNED) diag_run4(p, x, dc, row0 + g, min(4, nr - g), acc);   // only hybrid plans have shapes
#pragma unroll
    for (int w = 0; w < kDirectW; ++w) {
        const int j = b[0] + w;
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (j >= b[u] && j < b[u + 1]) acc[u] += v[w];
    }
    for (int j = b[0] + kDirectW; j < e4; ++j) {               // runs with more words
        const float z = gather<SIGNED>(x, __ldg(p.cols + j));
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (j >= b[u] && j < b[u + 1]) acc[u] += z;
    }
    float *yr = y + row0 + g;
    if (g + 4 <= nr && (reinterpret_cast<uintptr_t>(yr) & 15) == 0) {
        *reinterpret_cast<float4 *>(yr) = make_float4(acc[0], acc[1], acc[2], acc[3]);
    } else {
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (g + u < nr) yr[u] = acc[u];
    }
}

// The run of rows [g, g + 4) (g a multiple of 4, all four rows inside the
// matrix, y 16-byte aligned): direct_run's terms and order without its edge
// handling, for the full tiles of the direct kernel.
template <bool SIGNED, bool POS = false>
__device__ __forceinline__ void direct_run_full(const DevPlan &p, int dc, const float *__restrict__ x,
                                                float *__restrict__ y, int g)
{
    constexpr int kDirectWFull = direct_w_full<SIGNED>();
    const int4 r4 = __ldg(reinterpret_cast<const int4 *>(p.rowptr + g));
    const int e4 = __ldg(p.rowptr + g + 4);
    const int b[5] = {r4.x, r4.y, r4.z, r4.w, e4};
    int c[kDirectWFull];
#pragma unroll
    for (int w = 0; w < kDirectWFull; ++w) c[w] = b[0] + w < e4 ? __ldg(p.cols + b[0] + w) : 0;
    wait_prior_grid(x, y);
    float v[kDirectWFull];
#pragma unroll
    for (int w = 0; w < kDirectWFull; ++w) v[w] = gather_pos<SIGNED, POS>(x, c[w]);   // past the run: x[0], not added
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    if (SIGNED && p.dn == 1) {
        // one dense diagonal: which rows have its term comes from the launch
        // parameters (no plan reads on the chain); the terms and order of
        // diag_run4
        const int lo = p.d_lo[0], hi = p.d_hi[0], col = p.d_col[0];
        const float *xd = x + g + col;
        if (g >= lo && g + 4 <= hi && (col & 3) == 0) {   // x is 16-byte aligned
            float d[4];
            asm("ld.global.v4.f32 {%0, %1, %2, %3}, [%4];"
                : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3]) : "l"(xd));
#pragma unroll
            for (int u = 0; u < 4; ++u) acc[u] += d[u];
        } else {
            float d[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) d[u] = g + u >= lo && g + u < hi ? ldx(xd + u) : 0.f;
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (g + u >= lo && g + u < hi) acc[u] += d[u];
        }
    } else if (SIGNED) {
        diag_run4(p, x, dc, g, 4, acc);
    }
#pragma unroll
    for (int w = 0; w < kDirectWFull; ++w)
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (b[0] + w >= b[u] && b[0] + w < b[u + 1]) acc[u] += v[w];
    for (int j = b[0] + kDirectWFull; j < e4; ++j) {
        const float z = gather_pos<SIGNED, POS>(x, __ldg(p.cols + j));
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (j >= b[u] && j < b[u + 1]) acc[u] += z;
    }
    *reinterpret_cast<float4 *>(y + g) = make_float4(acc[0], acc[1], acc[2], acc[3]);
}

// direct_run_full with the tile's CSR words already in shared memory: ws[k]
// = cols[base + k] for k < lim (the words past lim, if any, from global
// memory).  The row pointers r4 / e4 of the run were loaded by the caller.
template <bool SIGNED>
__device__ __forceinline__ void direct_run_staged(const DevPlan &p, int dc, const float *__restrict__ x,
                                                  float *__restrict__ y, int g, int4 r4, int e4,
                                                  const int *ws, int base, int lim)
{
    const int b[5] = {r4.x, r4.y, r4.z, r4.w, e4};
    int c[kDirectW];
#pragma unroll
    for (int w = 0; w < kDirectW; ++w) {
        const int j = b[0] + w;
        c[w] = j < e4 ? (j - base < lim ? ws[j - base] : __ldg(p.cols + j)) : 0;
    }
    wait_prior_grid(x, y);
    float v[kDirectW];
#pragma unroll
    for (int w = 0; w < kDirectW; ++w) v[w] = b[0] + w < e4 ? gather<SIGNED>(x, c[w]) : 0.f;
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    if (SIGNED) diag_run4(p, x, dc, g, 4, acc);
#pragma unroll
    for (int w = 0; w < kDirectW; ++w)
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (b[0] + w >= b[u] && b[0] + w < b[u + 1]) acc[u] += v[w];
    for (int j = b[0] + kDirectW; j < e4; ++j) {
        const float z = gather<SIGNED>(x, j - base < lim ? ws[j - base] : __ldg(p.cols + j));
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (j >= b[u] && j < b[u + 1]) acc[u] += z;
    }
    *reinterpret_cast<float4 *>(y + g) = make_float4(acc[0], acc[1], acc[2], acc[3]);
}

template <bool SIGNED>
__device__ __forceinline__ void direct_run(const DevPlan &p, const Tile &t, const float *__restrict__ x,
                                           float *__restrict__ y, bool wait, int g)
{
    direct_run<SIGNED>(p, t.row0, tile_nrows(t), tile_dclass(t), x, y, wait, g);
}

// A direct tile in a 256-thread CTA: one pass (TILE_DIRECT4) or four
// (TILE_DIRECT_WIDE).
template <bool SIGNED>
__device__ __forceinline__ void tile_direct(const DevPlan &p, const Tile &t, const float *__restrict__ x,
                                            float *__restrict__ y, bool wait)
{
    const int passes = tile_kind(t) == TILE_DIRECT_WIDE ? kDirectWideRows / kDirectRows : 1;
    for (int k = 0; k < passes; ++k) direct_run<SIGNED>(p, t, x, y, wait && k == 0, 4 * (threadIdx.x + k * kBlock));
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
    if (!waited) { wait_prior_grid(x, y); waited = true; }
    const int r = t.row0;
    if (p.dia_shapes > 0 && r >= p.row_start && r < p.row_stop)
        for (int s = 0; s < p.dia_shapes; ++s) {
            const int4 sh = __ldg(p.shapes + s);
            if (r < sh.x || r >= sh.y) continue;
            const int2 dr = __ldg(p.shape_dias + s);
            for (int n = dr.x + tid; n < dr.y; n += kBlock) {
                const int c = r - sh.x + sh.z + __ldg(p.offsets + n);
                if (c >= sh.z && c < sh.z + sh.w) acc += ldx(x + c);
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
    case TILE_MERGE: tile_merge<SIGNED>(p, t, src, x, y, wait); break;
    case TILE_STREAM: tile_stream<SIGNED>(p, t, x, y, wait); break;
    case TILE_STREAM4: tile_stream4<SIGNED>(p, t, x, y, wait); break;
    case TILE_DIRECT4:
    case TILE_DIRECT_WIDE: tile_direct<SIGNED>(p, t, x, y, wait); break;
    case TILE_L1: tile_rows_seq<SIGNED>(p, t, src, x, y, wait); break;
    case TILE_L2: tile_rows<SIGNED, 2>(p, t, src, x, y, wait); break;
    case TILE_L4: tile_rows<SIGNED, 4>(p, t, src, x, y, wait); break;
    case TILE_L8: tile_rows<SIGNED, 8>(p, t, src, x, y, wait); break;
    case TILE_L16: tile_rows<SIGNED, 16>(p, t, src, x, y, wait); break;
    case TILE_L32: tile_rows<SIGNED, 32>(p, t, src, x, y, wait); break;
    default: long_row<SIGNED>(p, t, x, y, wait); break;
    }
}

// The tile kinds of a stream plan (tile_mode 2 without lane tiles): kernels
// that only ever see these carry no lane-tile code and fit more CTAs per SM.
template <bool SIGNED>
__device__ __forceinline__ void run_lean_tile(const DevPlan &p, const Tile &t, const float *__restrict__ x,
                                              float *__restrict__ y, bool wait)
{
    switch (tile_kind(t)) {
    case TILE_STREAM4: tile_stream4<SIGNED>(p, t, x, y, wait); break;
    case TILE_STREAM: tile_stream<SIGNED>(p, t, x, y, wait); break;
    case TILE_DIRECT4:
    case TILE_DIRECT_WIDE: tile_direct<SIGNED>(p, t, x, y, wait); break;
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

// Work items of the batch and served launches (256-thread CTAs): a wide
// direct tile is four items, part k holding its rows [1024 k, 1024 k + 1024)
// (every thread one run, all loads of the item in flight); any other tile is
// one item (part 0).
__host__ __device__ inline int tile_parts(int per_tile) { return per_tile == 3 ? kDirectWideRows / kDirectRows : 1; }

template <bool SIGNED, bool LEAN>
__device__ __forceinline__ void run_tile_part(const DevPlan &p, const Tile &t, int part,
                                              const float *__restrict__ x, float *__restrict__ y, bool wait)
{
    const bool wide = tile_kind(t) == TILE_DIRECT_WIDE;
    if (threadIdx.x == 0) {
        const int r = wide ? kDirectRows * part : 0;
        prefetch_x_window(x, p.N, t.row0 + r, wide ? min(kDirectRows, tile_nrows(t) - r) : tile_nrows(t));
    }
    if (wide) direct_run<SIGNED>(p, t, x, y, wait, 4 * (threadIdx.x + kBlock * part));
    else if (LEAN) run_lean_tile<SIGNED>(p, t, x, y, wait);
    else run_tile<SIGNED>(p, t, x, y, wait);
}

}  // namespace tc
