// tc_tile.cuh -- device code of one multiply tile, shared by the single-plan
// kernel (tc_spmv.cu) and the multi-plan persistent kernel (tc_batch.cu) so
// that a matrix gets bit-identical y alone and inside a batch.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "tc_internal.h"

namespace tc {

// Shared memory of the tile kernel: row pointers, per-row sums, and one
// buffer that first holds the tile's gathered CSR terms and then the x window
// of a dense diagonal shape (the two are never live at the same time).
__host__ __device__ inline int smem_rp_ints(int rows_cap) { return (rows_cap + 8 + 3) & ~3; }
// per-row sums; at least one slot per warp for the long-row reduction
__host__ __device__ inline int smem_racc_floats(int rows_cap) { return ((rows_cap < 32 ? 32 : rows_cap) + 3) & ~3; }
__host__ __device__ inline int smem_buf_floats(int rows_cap, int nnz_cap, int max_span)
{
    int xw = rows_cap + max_span + 16;
    int b = nnz_cap > xw ? nnz_cap : xw;
    return (b + 3) & ~3;
}

inline size_t spmv_smem_bytes_impl(int rows_cap, int nnz_cap, int max_span)
{
    return sizeof(int) * (size_t)smem_rp_ints(rows_cap) + sizeof(float) * (size_t)smem_racc_floats(rows_cap) +
           sizeof(float) * (size_t)smem_buf_floats(rows_cap, nnz_cap, max_span) + 16;
}


constexpr int kU = 8;   // loads in flight per thread per staging round

template <bool SIGNED>
__device__ __forceinline__ float gather(const float *__restrict__ x, int c)
{
    if (SIGNED) {
        float v = __ldg(x + (c >> 1));
        return (c & 1) ? v : -v;
    }
    return __ldg(x + c);
}

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Adds the dense-diagonal terms of rows [r0, r0+nr) of one tile to racc[] (in
// shared memory), staging each shape's x window in xw[].  All threads call.
__device__ __forceinline__ void tile_diagonals(const DevPlan &p, const float *__restrict__ x,
                                               int r0, int nr, float *racc, float *xw)
{
    const int tid = threadIdx.x;
    const int r1 = r0 + nr;
    if (r1 <= p.row_start || r0 >= p.row_stop) return;
    for (int s = 0; s < p.dia_shapes; ++s) {
        const int4 sh = __ldg(p.shapes + s);     // xStart, xStop, yStart, Msub
        const int ra = max(r0, sh.x), rb = min(r1, sh.y);
        if (ra >= rb) continue;                  // uniform across the CTA
        const int2 dr = __ldg(p.shape_dias + s);
        const int omin = __ldg(p.offsets + dr.x), omax = __ldg(p.offsets + dr.y - 1);
        const int cbase = sh.z - sh.x;           // col = row + cbase + off
        int lo = ra + cbase + omin, hi = rb - 1 + cbase + omax;   // inclusive
        lo = max(lo, sh.z);
        hi = min(hi, sh.z + sh.w - 1);
        if (lo <= hi) {
            // x[lo..hi] -> xw[0..]; 16-byte loads on the aligned interior.
            const int a4 = (lo + 3) & ~3, b4 = (hi + 1) & ~3;   // [a4, b4) aligned
            const bool x16 = (reinterpret_cast<uintptr_t>(x) & 15) == 0;
            if (x16 && a4 < b4) {
                const float4 *x4 = reinterpret_cast<const float4 *>(x + a4);
                const int n4 = (b4 - a4) >> 2;
                for (int i = tid; i < n4; i += kBlock) {
                    float4 v = __ldg(x4 + i);
                    float *d = xw + (a4 - lo) + 4 * i;
                    d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
                }
                for (int i = lo + tid; i < a4; i += kBlock) xw[i - lo] = __ldg(x + i);
                for (int i = b4 + tid; i <= hi; i += kBlock) xw[i - lo] = __ldg(x + i);
            } else {
                for (int i = lo + tid; i <= hi; i += kBlock) xw[i - lo] = __ldg(x + i);
            }
        }
        __syncthreads();
        if (lo <= hi) {
            for (int r = ra + tid; r < rb; r += kBlock) {
                float acc = racc[r - r0];
                const int cb = r + cbase;
                for (int n = dr.x; n < dr.y; ++n) {
                    const int c = cb + __ldg(p.offsets + n);
                    if (c >= lo && c <= hi) acc += xw[c - lo];
                }
                racc[r - r0] = acc;
            }
        }
        __syncthreads();
    }
}

template <bool SIGNED>
__device__ void long_row(const DevPlan &p, const Tile &t, const float *__restrict__ x,
                         float *__restrict__ y, float *red)
{
    const int tid = threadIdx.x;
    const int *__restrict__ cols = p.cols + t.nz0;
    float acc = 0.f;
    for (int base = 0; base < t.nnz; base += kBlock * kU) {
        int c[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            int i = base + u * kBlock + tid;
            c[u] = i < t.nnz ? __ldg(cols + i) : -1;
        }
#pragma unroll
        for (int u = 0; u < kU; ++u)
            if (c[u] >= 0) acc += gather<SIGNED>(x, c[u]);
    }
    acc = warp_sum(acc);
    if ((tid & 31) == 0) red[tid >> 5] = acc;
    __syncthreads();
    if (tid < 32) {
        float v = tid < kBlock / 32 ? red[tid] : 0.f;
        v = warp_sum(v);
        if (tid == 0) {
            const int r = t.row0;
            if (p.dia_shapes > 0 && r >= p.row_start && r < p.row_stop) {
                for (int s = 0; s < p.dia_shapes; ++s) {
                    const int4 sh = __ldg(p.shapes + s);
                    if (r < sh.x || r >= sh.y) continue;
                    const int2 dr = __ldg(p.shape_dias + s);
                    for (int n = dr.x; n < dr.y; ++n) {
                        int col = r - sh.x + sh.z + __ldg(p.offsets + n);
                        if (col >= sh.z && col < sh.z + sh.w) v += __ldg(x + col);
                    }
                }
            }
            y[r] = v;
        }
    }
}

// Processes one tile (any kind).  Shared by the single-plan and the batched
// kernels so a matrix gives bit-identical y alone and inside a batch.
template <bool SIGNED>
__device__ void run_tile(const DevPlan &p, const Tile &t, const float *__restrict__ x,
                         float *__restrict__ y, char *smem)
{
    const int tid = threadIdx.x;
    int *rp = reinterpret_cast<int *>(smem);
    float *racc = reinterpret_cast<float *>(rp + smem_rp_ints(p.rows_cap));
    float *vals = racc + smem_racc_floats(p.rows_cap);
    float *xw = vals;   // reused once the CSR terms are summed
    const int kind = tile_kind(t);
    if (kind == TILE_LONG) {
        long_row<SIGNED>(p, t, x, y, racc);
        return;
    }
    const int nr = tile_nrows(t), nz = t.nnz, r0 = t.row0, nz0 = t.nz0;

    // Phase A: row pointers and CSR entries of the tile, loads batched so
    // that each thread keeps kU requests in flight.
    {
        int v[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            int i = u * kBlock + tid;
            v[u] = i <= nr ? __ldg(p.rowptr + r0 + i) : 0;
        }
        for (int base = 0; base < nz; base += kBlock * kU) {
            int c[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                int i = base + u * kBlock + tid;
                c[u] = i < nz ? __ldg(p.cols + nz0 + i) : 0;
            }
            float g[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                int i = base + u * kBlock + tid;
                g[u] = i < nz ? gather<SIGNED>(x, c[u]) : 0.f;
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                int i = base + u * kBlock + tid;
                if (i < nz) vals[i] = g[u];
            }
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            int i = u * kBlock + tid;
            if (i <= nr) rp[i] = v[u] - nz0;
        }
    }
    __syncthreads();

    // Phase B: per-row sums of the staged entries.
    if (kind == TILE_SCALAR) {
        for (int r = tid; r < nr; r += kBlock) {
            float s = 0.f;
            const int e = rp[r + 1];
            for (int j = rp[r]; j < e; ++j) s += vals[j];
            racc[r] = s;
        }
    } else {
        const int lane = tid & 31, warp = tid >> 5;
        for (int r = warp; r < nr; r += kBlock / 32) {
            float s = 0.f;
            const int e = rp[r + 1];
            for (int j = rp[r] + lane; j < e; j += 32) s += vals[j];
            s = warp_sum(s);
            if (lane == 0) racc[r] = s;
        }
    }
    __syncthreads();

    // Phase C: dense diagonals, then one coalesced store of y.
    if (p.dia_shapes > 0) tile_diagonals(p, x, r0, nr, racc, xw);
    for (int r = tid; r < nr; r += kBlock) y[r0 + r] = racc[r];
}

}  // namespace tc
