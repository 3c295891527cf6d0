// tc_spmv.cu -- the multiply: tile planner, device format upload, and the
// value-free hybrid SpMV / SpMM kernels for sm_100a.
//
// Replaces taichi_SpMV's dispatch and kernels (TaiChi.cu:965-1329).  The
// reference launches one of four CSR-vector kernels with a single vector
// width per matrix (TPV = sqrt of the mean row length) and a volatile
// shared-memory reduction.  Here the host planner cuts the rows into tiles
// and gives each tile its own lanes-per-row from that tile's row lengths (a
// CTA per row above a length limit); the kernel walks the tile list, keeps
// kRPT rows' loads in flight per lane group, adds the dense-diagonal terms in
// registers and writes y once with warp-shuffle reductions.  Launches use
// programmatic dependent launch so the next multiply's index loads overlap
// the previous one's tail.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "tc_internal.h"
#include "tc_tile.cuh"
#include "tc_tma.cuh"

namespace tc {

// ------------------------------------------------------------------ planner
// Lanes per row from the mean row length of a run of rows: one lane per row
// until rows average more than 16 entries, then the smallest power of two
// giving each lane about 8 entries, capped at max_lanes.  (The CSR words come
// from shared memory, so a thread walking its own row costs no coalescing.)
static int lanes_for(double mean, int max_lanes)
{
    if (mean <= 16.0) return 1;
    int l = 1;
    while (l < max_lanes && 8.0 * l < mean) l <<= 1;
    return l;
}

static int kind_of(int lanes)
{
    int k = 0;
    while ((1 << k) < lanes) ++k;
    return k;
}

int wide_tile_rows(int M, const tc_params &prm, int sms)
{
    if ((prm.flags & TC_FLAG_WIDE_FIXED) || sms <= 0) return kDirectWideRows;
    // two tiles per SM: every SM holds two CTAs of the same size
    const long per = ((long)M + 2L * sms - 1) / (2L * sms);
    return (int)std::min<long>(kDirectWideRows, std::max<long>(kDirectRows, (per + 3) & ~3L));
}

void plan_tiles(const int *rp, int M, const tc_params &prm, int min_tiles, std::vector<Tile> &tiles,
                int *nvec, int *nlong)
{
    const int spread = (int)std::min<int64_t>(kStreamNnz, std::max<int64_t>(512, (int64_t)rp[M] / std::max(1, min_tiles)));
    const int long_len = std::max(1, std::min(prm.tile_nnz, kStageNnz));
    const int rows_cap = std::max(1, std::min(prm.tile_rows, kMaxTileRows));
    tiles.clear();
    *nvec = *nlong = 0;
    if (prm.tile_mode == 2 && prm.tile_rows >= kDirectRows &&
        !(prm.flags & (TC_FLAG_NO_DIRECT | TC_FLAG_NO_WIDE | TC_FLAG_ROWS_STRIDED)) && M >= kDirectWideRows &&
        rp[M] <= M) {
        // rows of at most one entry on average and none long: the whole
        // matrix as wide direct tiles (one 1024-thread CTA per 4096 rows)
        bool short_rows = true;
        for (int i = 0; i < M && short_rows; ++i) short_rows = rp[i + 1] - rp[i] <= kStreamRowMax;
        if (short_rows) {
            const int R = wide_tile_rows(M, prm, min_tiles / 4);
            for (int r = 0; r < M; r += R) {
                const int n = std::min(R, M - r);
                tiles.push_back(Tile{r, rp[r], rp[r + n] - rp[r], tile_word(n, TILE_DIRECT_WIDE)});
            }
            return;
        }
    }
    int r = 0;
    while (r < M) {
        if (rp[r + 1] - rp[r] > long_len) {
            tiles.push_back(Tile{r, rp[r], rp[r + 1] - rp[r], tile_word(1, TILE_LONG)});
            ++*nlong;
            ++r;
            continue;
        }
        if (prm.tile_mode == 2 && rp[r + 1] - rp[r] <= kStreamRowMax) {
            // stream tile: short rows up to the row and entry caps.  A run
            // that starts on a multiple of 4 rows and holds many rows runs 4
            // consecutive rows per thread: read directly from global memory
            // when they average at most one entry (TILE_DIRECT4), through
            // shared memory when at most two (TILE_STREAM4); otherwise one
            // row per thread (TILE_STREAM)
            const bool a4 = (r & 3) == 0 && !(prm.flags & TC_FLAG_ROWS_STRIDED);
            const int cap_rows = std::min(rows_cap, a4 ? kDirectRows : kStreamRows);
            const int cap_nnz = std::max(1, std::min(2 * prm.tile_nnz, spread));
            int n = 0;
            while (r + n < M && n < cap_rows && rp[r + n + 1] - rp[r + n] <= kStreamRowMax &&
                   rp[r + n + 1] - rp[r] <= cap_nnz)
                ++n;
            if (n == 0) n = 1;        // a single row longer than cap_nnz but <= kStreamRowMax
            const int ent = rp[r + n] - rp[r];
            const bool direct = a4 && n >= 2 * kBlock && ent <= n && !(prm.flags & TC_FLAG_NO_DIRECT);
            const bool four = !direct && a4 && n >= 2 * kBlock && ent <= 2 * n;
            if (!direct) n = std::min(n, four ? kStream4Rows : kStreamRows);
            if (r + n < M) {          // end on a multiple of 256 rows (whole row sweeps), else of 4
                const int cut = (r + n) & ~255;
                if (cut - r >= 256) n = cut - r;
                else if (n > 4) n -= (r + n) & 3;
            }
            const int kind = direct ? TILE_DIRECT4 : four ? TILE_STREAM4 : TILE_STREAM;
            tiles.push_back(Tile{r, rp[r], rp[r + n] - rp[r], tile_word(n, kind)});
            r += n;
            continue;
        }
        // candidate run: up to 1024 rows (merge tiles: tile_rows), stopping
        // before a long row (stream mode: before a short row too)
        const int run_cap = prm.tile_mode == 0 ? std::min(rows_cap, kMergeRows) : 1024;
        int n = 0;
        while (r + n < M && n < run_cap && rp[r + n + 1] - rp[r + n] <= long_len &&
               !(prm.tile_mode == 2 && rp[r + n + 1] - rp[r + n] <= kStreamRowMax))
            ++n;
        if (prm.tile_mode == 0) {          // merge tile: rows + entries split evenly
            int rows = n;
            while (rows > 1 && rp[r + rows] - rp[r] > kStageNnz) rows = (rows + 1) / 2;
            tiles.push_back(Tile{r, rp[r], rp[r + rows] - rp[r], tile_word(rows, TILE_MERGE)});
            r += rows;
            continue;
        }
        int lanes = lanes_for((double)(rp[r + n] - rp[r]) / n, prm.max_lanes);
        int rows = std::min(std::min(n, tile_rows_for(lanes)), rows_cap);
        while (rows > 1 && rp[r + rows] - rp[r] > kStageNnz) rows = (rows + 1) / 2;   // fits a stage
        lanes = lanes_for((double)(rp[r + rows] - rp[r]) / rows, prm.max_lanes);
        if (lanes > 1) ++*nvec;
        tiles.push_back(Tile{r, rp[r], rp[r + rows] - rp[r], tile_word(rows, kind_of(lanes))});
        r += rows;
    }
}

// ------------------------------------------------------------------ kernels
namespace {

// Issues the copies of tile t into stage s (thread 0 only).
__device__ __forceinline__ void stage_tile(const DevPlan &p, int t, int *rp_buf, int *cw_buf,
                                           uint64_t *bar)
{
    if (t >= p.ntiles) return;
    const Tile tile = p.tiles[t];
    if (tile_kind(tile) == TILE_LONG || tile_kind(tile) >= TILE_STREAM) return;   // read from global
    const Window wr = window_of(tile.row0, (long)tile.row0 + tile_nrows(tile) + 1);
    const Window wc = window_of(tile.nz0, (long)tile.nz0 + tile.nnz);
    const unsigned br = (unsigned)(wr.b - wr.a), bc = tile.nnz ? (unsigned)(wc.b - wc.a) : 0u;
    mbar_expect_tx(bar, br + bc);
    bulk_load(rp_buf, reinterpret_cast<const char *>(p.rowptr) + wr.a, br, bar);
    if (bc) bulk_load(cw_buf, reinterpret_cast<const char *>(p.cols) + wc.a, bc, bar);
}

// The multiply: a persistent grid; each CTA walks tiles blockIdx.x,
// blockIdx.x + gridDim.x, ... with a two-stage pipeline: while one tile is
// processed from shared memory, the TMA engine brings in the row pointers
// and CSR words of the tile after next.  Rows longer than a stage are read
// straight from global memory (TILE_LONG).
template <bool SIGNED>
__global__ void __launch_bounds__(kBlock) spmv_tiles_kernel(DevPlan p, const float *__restrict__ x,
                                                            float *__restrict__ y)
{
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem);
    int *const buf = reinterpret_cast<int *>(smem + 16);
    const int stride = p.stage_rp + p.stage_cw;          // ints per stage
    allow_next_grid();
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        stage_tile(p, blockIdx.x, buf, buf + p.stage_rp, bar);
        stage_tile(p, blockIdx.x + gridDim.x, buf + stride, buf + stride + p.stage_rp, bar + 1);
    }
    unsigned phases = 0u;                                // bit s: parity of stage s
    bool waited = false;
    int i = 0;
    for (int t = blockIdx.x; t < p.ntiles; t += gridDim.x, ++i) {
        const int s = i & 1;
        int *const rp_s = buf + s * stride;
        int *const cw_s = rp_s + p.stage_rp;
        const Tile tile = p.tiles[t];
        if (tile_kind(tile) == TILE_LONG || tile_kind(tile) >= TILE_STREAM) {
            run_tile<SIGNED>(p, tile, x, y, !waited);
        } else {
            const bool ok = mbar_wait(bar + s, (phases >> s) & 1u);
            if (!__syncthreads_and(ok)) {          // every thread takes the same branch
                if (threadIdx.x == 0) atomicExch(p.err, 1);
                mbar_wait(bar + (s ^ 1), (phases >> (s ^ 1)) & 1u);   // copies in flight land
                return;
            }
            phases ^= 1u << s;
            const Window wr = window_of(tile.row0, 0), wc = window_of(tile.nz0, 0);
            const SharedSrc src{rp_s + wr.shift, cw_s + wc.shift, tile.nz0};
            run_tile_src<SIGNED>(p, tile, src, x, y, !waited);
        }
        waited = true;
        after_wait(x, y);                 // later tiles' x / y accesses follow the first tile's wait
        __syncthreads();                  // stage s is free again
        if (threadIdx.x == 0) {
            fence_async_shared();
            stage_tile(p, t + 2 * gridDim.x, rp_s, cw_s, bar + s);
        }
    }
    if (!waited) wait_prior_grid();
}

// The multiply of a plan of wide direct tiles: one 1024-thread CTA per 4096
// rows, one run of 4 rows per thread.  Few CTAs (the block scheduler's launch
// cost grows with the CTA count) that all fit at once (2 per SM at 32
// registers), each holding 1024 independent load chains.
// (A variant that read a per-run descriptor -- 4 packed row lengths and the
// run's words padded to an int4, loaded together instead of row pointers then
// words -- measured slower on R-MAT, 7.35 against 5.9 µs, and was dropped.)
// FULL: every tile is whole (M a multiple of kDirectWideRows, N >= M) and x
// and y are 16-byte aligned, so each run takes the edge-free path and the x
// window is one aligned 16 KB prefetch; the launch picks it from those facts.
// (One kernel holding both paths behind a per-tile branch ran the full tiles
// 0.8 µs slower per R-MAT scale 20 multiply than this split.)
// POS (with SIGNED and FULL): every word of the plan is an addition (no
// holes in its dense diagonals), so the gathers skip the sign.  The FULL
// body: z0 / z1, when z0 >= 0, are the tile's CSR word range as the launch
// parameters give it (the prefetch of the words then goes out at once),
// otherwise thread 0 reads the range from the tile record first.
template <bool SIGNED, bool POS>
__device__ __forceinline__ void wide_full(const DevPlan &p, const float *__restrict__ x, float *__restrict__ y,
                                          int z0, int z1)
{
    const int row0 = blockIdx.x * p.wide_rows;
    const int nr = min(p.wide_rows, p.M - row0);
    const int dc = SIGNED && p.dn != 1 ? tile_dclass(p.tiles[blockIdx.x]) : kDiagNone;
    if (threadIdx.x == 0) {
        prefetch_l2(x + row0, (unsigned)nr * sizeof(float));
        if (z0 >= 0) {
            prefetch_span(p.cols, z0, z1);
        } else if (p.prefetch) {
            // the tile's CSR words, so that the runs' word loads, which wait
            // for their row pointers, find them in L2
            const Tile t = p.tiles[blockIdx.x];
            prefetch_span(p.cols, t.nz0, t.nz0 + t.nnz);
        }
    }
    if (4 * (int)threadIdx.x >= nr) {
        wait_prior_grid(x, y);
        return;
    }
    direct_run_full<SIGNED, POS>(p, dc, x, y, row0 + 4 * threadIdx.x);
}

template <bool SIGNED, bool FULL, bool POS = false>
__global__ void __launch_bounds__(kDirectWideBlock, 2) spmv_wide_kernel(DevPlan p, const float *__restrict__ x,
                                                                     float *__restrict__ y)
{
    allow_next_grid();
    // wide tiles are laid out in order, p.wide_rows rows each (the last one
    // may be shorter), so the rows are known without waiting for the tile
    // record; only the diagonal class comes from it (a one-diagonal plan
    // needs no tile record: the parameters say which rows have the term)
    if (FULL) {
        wide_full<SIGNED, POS>(p, x, y, -1, -1);
    } else {
        // the edge path (direct_run) has no one-diagonal shortcut: every plan's
        // diagonal terms come from the tile's class
        const int row0 = blockIdx.x * p.wide_rows;
        const int nr = min(p.wide_rows, p.M - row0);
        const int dc = SIGNED ? tile_dclass(p.tiles[blockIdx.x]) : kDiagNone;
        if (threadIdx.x == 0) prefetch_x_window(x, p.N, row0, nr);
        direct_run<SIGNED>(p, row0, nr, dc, x, y, true, 4 * threadIdx.x);
    }
}

// The whole-tile wide kernel with each tile's first CSR word in the launch
// parameters (plans of at most kWideParamTiles tiles): the prefetch of a
// tile's words into L2 goes out when the CTA starts, together with its
// row-pointer loads, instead of after a read of the tile record.
template <bool SIGNED, bool POS>
__global__ void __launch_bounds__(kDirectWideBlock, 2)
    spmv_wide_starts_kernel(DevPlan p, const __grid_constant__ WideStarts ws, const float *__restrict__ x,
                            float *__restrict__ y)
{
    allow_next_grid();
    wide_full<SIGNED, POS>(p, x, y, ws.nz[blockIdx.x], ws.nz[blockIdx.x + 1]);
}

// The multiply of a stream plan of short rows, one row per thread, read
// straight from global memory: no tile records, shared memory or barriers.
// A CTA runs kBlock consecutive rows (coalesced row pointers and y
// stores).  Each thread loads its row's first W words together
// (immutable plan data, before griddepcontrol.wait), then their gathers and
// its dense-diagonal terms together, and adds the diagonal terms (offset
// order), then the words (stored order), then any further words W at a
// time: the terms and order of tile_rows_seq, so y is bit-identical to the
// stream tiles'.  Consecutive lanes hold consecutive rows, so a warp's load
// of word w of its 32 rows touches the few cache lines holding those rows,
// and its later words hit L1.  Against the stream tiles it spends no
// instructions on parking terms in shared memory and no barrier waits.
template <bool SIGNED, int W>
__global__ void __launch_bounds__(kBlock, kRowsMinBlocks)
    spmv_rows_kernel(DevPlan p, const float *__restrict__ x, float *__restrict__ y)
{
    allow_next_grid();
    const int r = blockIdx.x * kBlock + threadIdx.x;
    // warp 0 also brings into L2 the x window of the strip and the operands
    // of the strip a wave later (thread 0; the other warps skip it whole)
    const bool lead = threadIdx.x < 32;
    const bool ahead = lead && blockIdx.x + p.ahead < gridDim.x;
    int za = 0, zb = 0;
    if (lead && threadIdx.x == 0) prefetch_x_window(x, p.N, r, kBlock);
    const int b = r < p.M ? __ldg(p.rowptr + r) : 0;
    const int e = r < p.M ? __ldg(p.rowptr + r + 1) : 0;
    if (ahead) {
        const int ra = (blockIdx.x + p.ahead) * kBlock;
        za = __ldg(p.rowptr + ra);
        zb = __ldg(p.rowptr + min(ra + kBlock, p.M));
    }
    int c[W];
#pragma unroll
    for (int w = 0; w < W; ++w) c[w] = b + w < e ? __ldg(p.cols + b + w) : 0;
    if (ahead && threadIdx.x == 0) {
        const int ra = (blockIdx.x + p.ahead) * kBlock;
        prefetch_rows_ahead(p, ra, min(ra + kBlock, p.M), za, zb);
    }
    wait_prior_grid(x, y);
    // every slot is loaded (a slot past the row holds word 0, a load of x[0]
    // that is never added): no branch around the gathers
    float v[W];
#pragma unroll
    for (int w = 0; w < W; ++w) v[w] = gather<SIGNED>(x, c[w]);
    float acc = 0.f;
    if (SIGNED && p.dgen) {
        acc = diag_row(p, x, r);
    } else if (SIGNED && p.dn <= 4) {
        // the plan's offsets in order, named by constant indices (operands
        // straight from the parameter bank); a row outside an offset's range
        // loads x[0] for it and does not add it
        float d[4];
        bool in[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            in[u] = u < p.dn && r >= p.d_lo[u] && r < p.d_hi[u];
            d[u] = ldx(x + (in[u] ? r + p.d_col[u] : 0));
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (in[u]) acc += d[u];
    } else if (SIGNED) {
#pragma unroll 1
        for (int i = 0; i < p.dn; i += 4) {                      // the plan's offsets in order
            float d[4];
            bool in[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                in[u] = i + u < p.dn && r >= p.d_lo[i + u] && r < p.d_hi[i + u];
                d[u] = in[u] ? ldx(x + r + p.d_col[i + u]) : 0.f;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (in[u]) acc += d[u];
        }
    }
#pragma unroll
    for (int w = 0; w < W; ++w)
        if (b + w < e) acc += v[w];
#pragma unroll 1
    for (int j = b + W; j < e; j += W) {                            // longer rows, W words at a time
        int cc[W];
        float vv[W];
#pragma unroll
        for (int u = 0; u < W; ++u) cc[u] = j + u < e ? __ldg(p.cols + j + u) : 0;
#pragma unroll
        for (int u = 0; u < W; ++u) vv[u] = gather<SIGNED>(x, cc[u]);
#pragma unroll
        for (int u = 0; u < W; ++u)
            if (j + u < e) acc += vv[u];
    }
    if (r < p.M) y[r] = acc;
}

// The multiply of a stream plan: one CTA per tile, no shared-memory stages
// (stream tiles read their CSR words as coalesced int4s; lane and long tiles
// read global memory directly).  LEAN: the plan holds only stream and long
// tiles, so the kernel carries no lane-tile code and fits more CTAs per SM.
template <bool SIGNED, bool LEAN>
__global__ void __launch_bounds__(kBlock, LEAN ? (SIGNED ? kLeanMinBlocksSigned : kLeanMinBlocks) : 1)
    spmv_grid_kernel(DevPlan p, const float *__restrict__ x, float *__restrict__ y)
{
    allow_next_grid();
    const Tile t = p.tiles[blockIdx.x];
    if (threadIdx.x == 0) prefetch_x_window(x, p.N, t.row0, tile_nrows(t));
    if (LEAN) {
        run_lean_tile<SIGNED>(p, t, x, y, true);
    } else {
        run_tile<SIGNED>(p, t, x, y, true);
    }
}

// The whole-tile wide kernel with the tiles' word bounds in the launch
// parameters: each CTA reads its tile's CSR words into shared memory with
// coalesced int4 loads issued together with its row-pointer loads, so the
// chain before the gathers is one memory round trip instead of two (row
// pointers, then the words they point to).  Same runs, terms and order as
// spmv_wide_kernel<SIGNED, true>.
template <bool SIGNED>
__global__ void __launch_bounds__(kDirectWideBlock, 2)
    spmv_wide_bounds_kernel(DevPlan p, const __grid_constant__ WideBounds tb, const float *__restrict__ x,
                            float *__restrict__ y)
{
    __shared__ int4 sw[kWideWordQ];
    allow_next_grid();
    const int row0 = blockIdx.x * kDirectWideRows;
    const int dc = SIGNED ? tile_dclass(p.tiles[blockIdx.x]) : kDiagNone;
    if (threadIdx.x == 0) prefetch_l2(x + row0, kDirectWideRows * sizeof(float));
    const int nz0 = tb.nz[blockIdx.x], nz1 = tb.nz[blockIdx.x + 1];
    const int base = nz0 & ~3;
    const int nq = min((nz1 - base + 3) >> 2, kWideWordQ);
    const int4 *cq = reinterpret_cast<const int4 *>(p.cols + base);
    for (int i = threadIdx.x; i < nq; i += kDirectWideBlock) sw[i] = __ldg(cq + i);
    const int g = row0 + 4 * threadIdx.x;
    const int4 r4 = __ldg(reinterpret_cast<const int4 *>(p.rowptr + g));
    const int e4 = __ldg(p.rowptr + g + 4);
    __syncthreads();
    direct_run_staged<SIGNED>(p, dc, x, y, g, r4, e4, reinterpret_cast<const int *>(sw), base, 4 * nq);
}

// The multiply of a plan of stream tiles only (meshes, banded and other
// matrices of short, even rows): the grid kernel with no code for the other
// tile kinds.  MANY: more tiles than one wave, compiled for 8 CTAs per SM.
template <bool SIGNED, bool MANY>
__global__ void __launch_bounds__(kBlock, MANY ? kStreamManyMinBlocks
                                               : (SIGNED ? kLeanMinBlocksSigned : kLeanMinBlocks))
    spmv_stream_kernel(DevPlan p, const float *__restrict__ x, float *__restrict__ y)
{
    allow_next_grid();
    const Tile t = p.tiles[blockIdx.x];
    if (threadIdx.x == 0) {
        prefetch_x_window(x, p.N, t.row0, tile_nrows(t));
        if (MANY && blockIdx.x + p.ahead < p.ntiles) {   // the tile a wave later
            const Tile a = p.tiles[blockIdx.x + p.ahead];
            prefetch_rows_ahead(p, a.row0, a.row0 + tile_nrows(a), a.nz0, a.nz0 + a.nnz);
        }
    }
    tile_stream<SIGNED>(p, t, x, y, true);
}

// SpMM: a warp owns kRPW consecutive rows at a time; lane l holds columns
// [l*V, l*V+V) of the k right-hand sides, so every X / Y row access is one
// coalesced warp transaction.  The entries of the kRPW rows are walked in
// rounds (one entry per row per round) so their X-row loads overlap.
constexpr int kRPW = 4;

template <int V>
__device__ __forceinline__ void axpy_row(float (&acc)[V], const float *__restrict__ X, long off,
                                         int c0, int k, float sg)
{
    const float *xr = X + off + c0;
    if (V == 2 && c0 + 1 < k && ((reinterpret_cast<uintptr_t>(xr) & 7) == 0)) {
        const float2 v = __ldg(reinterpret_cast<const float2 *>(xr));
        acc[0] += sg * v.x;
        acc[V - 1] += sg * v.y;
    } else {
#pragma unroll
        for (int v = 0; v < V; ++v)
            if (c0 + v < k) acc[v] += sg * __ldg(xr + v);
    }
}

template <bool SIGNED, int V>
__global__ void __launch_bounds__(kBlock) spmm_rows_kernel(DevPlan p, const float *__restrict__ X,
                                                           int ldx, int k, float *__restrict__ Y,
                                                           int ldy)
{
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * kBlock + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * kBlock) >> 5;
    const int c0 = lane * V;
    const bool active = c0 < k;
    for (long r0l = (long)warp * kRPW; r0l < p.M; r0l += (long)nwarps * kRPW) {
        const int r0 = (int)r0l;
        // row pointers of the kRPW rows: lanes 0..nrow hold rowptr[r0 + lane]
        const int nrow = min(kRPW, p.M - r0);
        const int rpv = lane <= nrow ? __ldg(p.rowptr + r0 + lane) : 0;
        int rb[kRPW], re[kRPW];
#pragma unroll
        for (int q = 0; q < kRPW; ++q) {
            rb[q] = __shfl_sync(0xffffffffu, rpv, q);
            const int e = __shfl_sync(0xffffffffu, rpv, q + 1);
            re[q] = q < nrow ? e : rb[q];
        }
        float acc[kRPW][V];
#pragma unroll
        for (int q = 0; q < kRPW; ++q)
#pragma unroll
            for (int v = 0; v < V; ++v) acc[q][v] = 0.f;
        for (int t = 0;; ++t) {
            bool any = false;
            int cv[kRPW];
#pragma unroll
            for (int q = 0; q < kRPW; ++q) {
                const int j = rb[q] + t;
                cv[q] = j < re[q] ? __ldg(p.cols + j) : -1;
                any |= cv[q] >= 0;
            }
            if (!any) break;            // uniform: every lane sees the same rows
#pragma unroll
            for (int q = 0; q < kRPW; ++q) {
                if (cv[q] < 0 || !active) continue;
                const int col = SIGNED ? (cv[q] >> 1) : cv[q];
                const float sg = (!SIGNED || (cv[q] & 1)) ? 1.f : -1.f;
                axpy_row<V>(acc[q], X, (long)col * ldx, c0, k, sg);
            }
        }
        if (p.dia_shapes > 0) {
#pragma unroll
            for (int q = 0; q < kRPW; ++q) {
                const int r = r0 + q;
                if (q >= nrow || r < p.row_start || r >= p.row_stop || !active) continue;
                for (int s = 0; s < p.dia_shapes; ++s) {
                    const int4 sh = __ldg(p.shapes + s);
                    if (r < sh.x || r >= sh.y) continue;
                    const int2 dr = __ldg(p.shape_dias + s);
                    for (int n = dr.x; n < dr.y; ++n) {
                        const int col = r - sh.x + sh.z + __ldg(p.offsets + n);
                        if (col >= sh.z && col < sh.z + sh.w)
                            axpy_row<V>(acc[q], X, (long)col * ldx, c0, k, 1.f);
                    }
                }
            }
        }
        if (active) {
#pragma unroll
            for (int q = 0; q < kRPW; ++q) {
                if (q >= nrow) continue;
                float *yr = Y + (long)(r0 + q) * ldy + c0;
                if (V == 2 && c0 + 1 < k && ((reinterpret_cast<uintptr_t>(yr) & 7) == 0)) {
                    *reinterpret_cast<float2 *>(yr) = make_float2(acc[q][0], acc[q][V - 1]);
                } else {
#pragma unroll
                    for (int v = 0; v < V; ++v)
                        if (c0 + v < k) yr[v] = acc[q][v];
                }
            }
        }
    }
}

int g_num_sms = 0;

int num_sms()
{
    if (g_num_sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
        if (g_num_sms <= 0) g_num_sms = 148;
    }
    return g_num_sms;
}

}  // namespace

size_t stream_smem_bytes(const DevPlan &dp)
{
    return 16 + 2 * sizeof(int) * (size_t)(dp.stage_rp + dp.stage_cw);
}

template <bool SIGNED>
static tc_status launch_tiles(const DevPlan &dp, const WideBounds *wb, const WideStarts *ws, const float *x,
                              float *y, cudaStream_t s)
{
    if (dp.ntiles <= 0) return TC_OK;
    const size_t smem = dp.per_tile ? 0 : stream_smem_bytes(dp);
    if (!dp.per_tile) TC_CHECK(ensure_smem((const void *)spmv_tiles_kernel<SIGNED>, smem));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(dp.per_tile ? dp.ntiles : dp.grid);
    cfg.blockDim = dim3(dp.per_tile == 3 ? kDirectWideBlock : kBlock);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = dp.pdl ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const bool full = dp.M % 4 == 0 && dp.N >= dp.M &&
                      ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15) == 0;
    if (dp.per_tile == 3 && full && wb && dp.wide_rows == kDirectWideRows && dp.M % kDirectWideRows == 0)
        TC_CUDA(cudaLaunchKernelEx(&cfg, spmv_wide_bounds_kernel<SIGNED>, dp, *wb, x, y));
    else if (dp.per_tile == 3 && full && ws && SIGNED && dp.pos)
        TC_CUDA(cudaLaunchKernelEx(&cfg, spmv_wide_starts_kernel<SIGNED, true>, dp, *ws, x, y));
    else if (dp.per_tile == 3 && full && ws)
        TC_CUDA(cudaLaunchKernelEx(&cfg, spmv_wide_starts_kernel<SIGNED, false>, dp, *ws, x, y));
    else if (dp.per_tile == 3 && full && SIGNED && dp.pos)
        TC_CUDA(cudaLaunchKernelEx(&cfg, spmv_wide_kernel<SIGNED, true, true>, dp, x, y));
    else if (dp.per_tile == 3 && full) TC_CUDA(cudaLaunchKernelEx(&cfg, spmv_wide_kernel<SIGNED, true>, dp, x, y));
    else if (dp.per_tile == 3) TC_CUDA(cudaLaunchKernelEx(&cfg, spmv_wide_kernel<SIGNED, false>, dp, x, y));
    else if (dp.per_tile == 4 && dp.rows) {
        cfg.gridDim = dim3((unsigned)((dp.M + kBlock - 1) / kBlock));
        if (dp.rows_w <= 4) TC_CUDA(cudaLaunchKernelEx(&cfg, spmv_rows_kernel<SIGNED, 4>, dp, x, y));
        else if (dp.rows_w <= 6) TC_CUDA(cudaLaunchKernelEx(&cfg, spmv_rows_kernel<SIGNED, 6>, dp, x, y));
        else TC_CUDA(cudaLaunchKernelEx(&cfg, spmv_rows_kernel<SIGNED, 8>, dp, x, y));
    }
    else if (dp.per_tile == 4 && dp.ntiles > kLeanMinBlocks * num_sms())
        TC_CUDA(cudaLaunchKernelEx(&cfg, spmv_stream_kernel<SIGNED, true>, dp, x, y));
    else if (dp.per_tile == 4) TC_CUDA(cudaLaunchKernelEx(&cfg, spmv_stream_kernel<SIGNED, false>, dp, x, y));
    else if (dp.per_tile == 2) TC_CUDA(cudaLaunchKernelEx(&cfg, spmv_grid_kernel<SIGNED, true>, dp, x, y));
    else if (dp.per_tile) TC_CUDA(cudaLaunchKernelEx(&cfg, spmv_grid_kernel<SIGNED, false>, dp, x, y));
    else TC_CUDA(cudaLaunchKernelEx(&cfg, spmv_tiles_kernel<SIGNED>, dp, x, y));
    return TC_OK;
}

tc_status launch_spmv(const DevPlan &dp, const float *x, float *y, cudaStream_t s, const WideBounds *wb,
                      const WideStarts *ws)
{
    if (dp.M == 0) return TC_OK;
    // no columns: no terms, and the kernels' unconditional loads of x[0]
    // (slots past a row's words) would have no x to read
    if (dp.N == 0) {
        TC_CUDA(cudaMemsetAsync(y, 0, sizeof(float) * (size_t)dp.M, s));
        return TC_OK;
    }
    if (dp.nwtiles > 0) return launch_window(dp, x, y, s);
    return dp.hybrid ? launch_tiles<true>(dp, wb, ws, x, y, s) : launch_tiles<false>(dp, wb, ws, x, y, s);
}

tc_status launch_plan(const tc_plan *p, const float *x, float *y, cudaStream_t s)
{
    if (!p->h_wide_nz.empty()) {
        WideBounds wb;
        memcpy(wb.nz, p->h_wide_nz.data(), sizeof(int) * p->h_wide_nz.size());
        return launch_spmv(p->dev_plan(), x, y, s, &wb, nullptr);
    }
    if (!p->h_wide_z.empty()) {
        WideStarts ws;
        memcpy(ws.nz, p->h_wide_z.data(), sizeof(int) * p->h_wide_z.size());
        return launch_spmv(p->dev_plan(), x, y, s, nullptr, &ws);
    }
    return launch_spmv(p->dev_plan(), x, y, s, nullptr, nullptr);
}

tc_status launch_spmm(const DevPlan &dp, const float *X, int ldx, int k, float *Y, int ldy,
                      cudaStream_t s)
{
    if (dp.M == 0) return TC_OK;
    const long warps = (dp.M + kRPW - 1) / kRPW;
    const int grid = (int)std::min<long>((warps + kBlock / 32 - 1) / (kBlock / 32), num_sms() * 16L);
    if (k <= 32) {
        if (dp.hybrid) spmm_rows_kernel<true, 1><<<grid, kBlock, 0, s>>>(dp, X, ldx, k, Y, ldy);
        else spmm_rows_kernel<false, 1><<<grid, kBlock, 0, s>>>(dp, X, ldx, k, Y, ldy);
    } else {
        if (dp.hybrid) spmm_rows_kernel<true, 2><<<grid, kBlock, 0, s>>>(dp, X, ldx, k, Y, ldy);
        else spmm_rows_kernel<false, 2><<<grid, kBlock, 0, s>>>(dp, X, ldx, k, Y, ldy);
    }
    TC_CUDA(cudaGetLastError());
    return TC_OK;
}

}  // namespace tc

// ------------------------------------------------------------- plan upload
tc::DevPlan tc_plan::dev_plan() const
{
    tc::DevPlan d{};
    d.rowptr = d_rowptr;
    d.cols = d_cols;
    d.tiles = d_tiles;
    d.shapes = d_shapes;
    d.shape_dias = d_shape_dias;
    d.offsets = d_offsets;
    d.M = M;
    d.N = N;
    d.ntiles = ntiles;
    d.dia_shapes = dia_shapes;
    d.row_start = row_start;
    d.row_stop = row_stop;
    d.hybrid = hybrid;
    d.max_span = max_span;
    d.pdl = (params.flags & TC_FLAG_NO_PDL) ? 0 : 1;
    d.stage_rp = stage_rp;
    d.stage_cw = stage_cw;
    d.grid = grid;
    d.per_tile = params.tile_mode != 2 ? 0
               : ntiles == 0 ? 2
               : ntiles_wide == ntiles ? 3
               : ntiles_stream == ntiles ? 4
               : ntiles_lanes == 0 ? 2 : 1;
    d.err = d_err;
    d.wide_rows = wide_rows;
    d.skew = stream_skew;
    d.dn = 0;
    d.dgen = 0;
    if (dia_shapes == 1 && num_negs <= tc::kPlanDiags && (int)h_offsets.size() >= num_negs) {
        // the rows where diag_row adds each offset's term (TaiChi.cu:1014-1023)
        const int xs = h_xStart[0], xe = h_xStop[0];
        d.dn = num_negs;
        for (int i = 0; i < num_negs; ++i) {
            const int off = h_offsets[i];
            d.d_lo[i] = std::max(xs + std::max(0, -off), row_start);
            d.d_hi[i] = std::min(xe - std::max(0, off), row_stop);
            d.d_col[i] = h_yStart[0] - xs + off;
        }
    } else if (dia_shapes > 0) {
        d.dgen = 1;
    }
    // the rows kernel: a stream plan (every row at most kStreamRowMax words)
    // of short rows, or any stream plan on request
    d.rows = 0;
    if (d.per_tile == 4 && !(params.flags & TC_FLAG_NO_ROWS))
        d.rows = (params.flags & TC_FLAG_ROWS) || (M > 0 && nnz_csr <= (int64_t)tc::kRowsMeanMax * M && tc::kRowsByDefault);
    d.rows_w = params.rows_w ? params.rows_w : rows_w;
    d.pos = hybrid && all_pos ? 1 : 0;
    // CTAs resident at once (the stream kernel's many-tile build, the rows
    // kernel): the CTA that starts when this one ends is about this far on
    d.prefetch = (params.flags & TC_FLAG_NO_PREFETCH) ? 0 : 1;
    d.ahead = (params.flags & TC_FLAG_NO_PREFETCH) ? (1 << 30)
            : (d.rows ? tc::kRowsMinBlocks : tc::kStreamManyMinBlocks) * tc::num_sms();
    d.wtiles = d_wtiles;
    d.nwtiles = nwtiles;
    d.wlo = wlo;
    d.whi = whi;
    d.w_rp = w_rp;
    d.w_cw = w_cw;
    d.w_xw = w_xw;
    d.w_stages = w_stages;
    d.w_grid = w_grid;
    return d;
}

int64_t tc_plan::spmv_bytes() const
{
    // 4(M+1) row pointers + 4 per CSR entry + x read once + y written once +
    // 20 bytes per shape descriptor + 4 per dense-diagonal offset.
    return 4LL * (M + 1) + 4LL * nnz_csr + 4LL * N + 4LL * M + 20LL * dia_shapes +
           4LL * num_negs;
}

namespace tc {

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// Diagonal class of rows [r0, r1) (see kDiagGeneral / kDiagNone): the
// multiply adds the dense-diagonal terms of such a tile without searching the
// shapes per row, with the same terms in the same order as diag_row.
static int diag_class(const tc_plan *p, int r0, int r1)
{
    if (p->dia_shapes == 0 || r1 <= p->row_start || r0 >= p->row_stop) return kDiagNone;
    int found = -1;
    for (int s = 0; s < p->dia_shapes; ++s) {
        if (r1 <= p->h_xStart[s] || r0 >= p->h_xStop[s]) continue;
        if (found >= 0) return kDiagGeneral;        // two shapes share rows of the tile
        found = s;
    }
    if (found < 0) return kDiagNone;
    const int xs = p->h_xStart[found], xe = p->h_xStop[found], msub = xe - xs;
    if (r0 < xs || r1 > xe || r0 < p->row_start || r1 > p->row_stop) return kDiagGeneral;
    for (int n = p->h_nDiasPtr[found]; n < p->h_nDiasPtr[found + 1]; ++n) {
        const int off = p->h_offsets[n];
        if (r0 - xs + off < 0 || r1 - 1 - xs + off >= msub) return kDiagGeneral;
    }
    return found + 1 < kDiagNone ? found + 1 : kDiagGeneral;
}

tc_status plan_upload(tc_plan *p, const int *csrRow, const int *csrCol, cudaStream_t stream)
{
    const int M = p->M;
    std::vector<Tile> tiles;
    plan_tiles(csrRow, M, p->params, 4 * num_sms(), tiles, &p->ntiles_vector, &p->ntiles_long);
    p->ntiles_lanes = 0;
    p->ntiles_wide = 0;
    p->ntiles_stream = 0;
    for (const Tile &t : tiles) {
        p->ntiles_wide += tile_kind(t) == TILE_DIRECT_WIDE;
        p->ntiles_stream += tile_kind(t) == TILE_STREAM;
    }
    // the direct kernel finds a wide tile's rows from its index
    for (size_t i = 0; i < tiles.size() && p->ntiles_wide; ++i)
        if (tiles[i].row0 != (int)i * tile_nrows(tiles[0]) || tile_kind(tiles[i]) != TILE_DIRECT_WIDE)
            return fail(TC_ERR_FORMAT, "wide tile %d out of order", (int)i);
    for (const Tile &t : tiles) {
        p->ntiles_lanes += tile_kind(t) <= TILE_L32 || tile_kind(t) == TILE_MERGE;
        if (tile_nrows(t) < 1 || tile_nrows(t) > kMaxTileNrows)
            return fail(TC_ERR_FORMAT, "tile of %d rows", tile_nrows(t));
    }
    p->ntiles = (int)tiles.size();
    p->nnz_csr = csrRow[M];
    p->wide_rows = p->ntiles_wide ? tile_nrows(tiles[0]) : kDirectWideRows;
    {   // the most common length of the rows stream tiles hold: skewed slots
        // when it is a multiple of 8 (see vslot), sampled rows
        std::vector<int> h(kStreamRowMax + 1, 0);
        const int step = std::max(1, M / 65536);
        for (int r = 0; r < M; r += step) {
            const int L = csrRow[r + 1] - csrRow[r];
            if (L <= kStreamRowMax) ++h[L];
        }
        const int mode = (int)(std::max_element(h.begin() + 1, h.end()) - h.begin());
        p->stream_skew = h[mode] > 0 && mode % 8 == 0;
        // a hybrid plan with no holes: every word adds its term
        p->all_pos = 1;
        if (p->hybrid)
            for (int64_t j = 0; j < csrRow[M] && p->all_pos; ++j) p->all_pos = csrCol[j] & 1;
        // the rows kernel loads W words of a row together: the least of 4, 6, 8
        // that holds 90 % of the rows whole
        int64_t tot = 0, upto = 0;
        for (int L = 0; L <= kStreamRowMax; ++L) tot += h[L];
        p->rows_w = 8;
        for (int L = 0, w = 4; L <= 8 && tot > 0; ++L) {
            upto += h[L];
            if (L == w) {
                if (upto * 10 >= tot * 9) {
                    p->rows_w = w;
                    break;
                }
                w += 2;
            }
        }
    }
    p->h_wide_nz.clear();
    if (p->ntiles_wide == p->ntiles && p->ntiles > 0 && p->ntiles <= kWideBoundTiles &&
        M % kDirectWideRows == 0 && (p->params.flags & TC_FLAG_WIDE_BOUNDS)) {
        for (const Tile &t : tiles) p->h_wide_nz.push_back(t.nz0);
        p->h_wide_nz.push_back(csrRow[M]);
    }
    // wide plans of few tiles: each tile's first word travels in the launch
    // parameters, for the word prefetch
    p->h_wide_z.clear();
    if (p->ntiles_wide == p->ntiles && p->ntiles > 0 && p->ntiles <= kWideParamTiles &&
        !(p->params.flags & (TC_FLAG_NO_PREFETCH | TC_FLAG_NO_PARAM_STARTS))) {
        for (const Tile &t : tiles) p->h_wide_z.push_back(t.nz0);
        p->h_wide_z.push_back(csrRow[M]);
    }
    // shared-memory stage sizes (ints, multiples of 4) from the largest tile
    int max_rows = 1, max_nnz = 0;
    for (const Tile &t : tiles)
        if (tile_kind(t) != TILE_LONG && tile_kind(t) < TILE_STREAM) {
            max_rows = std::max(max_rows, tile_nrows(t));
            max_nnz = std::max(max_nnz, t.nnz);
        }
    p->stage_rp = (max_rows + 1 + 8 + 3) & ~3;
    p->stage_cw = (max_nnz + 8 + 3) & ~3;

    // shape table {xStart, xStop, yStart, Msub} and offset ranges
    std::vector<int4> shapes(p->dia_shapes);
    std::vector<int2> sd(p->dia_shapes);
    p->max_span = 0;
    for (int s = 0; s < p->dia_shapes; ++s) {
        shapes[s] = make_int4(p->h_xStart[s], p->h_xStop[s], p->h_yStart[s],
                              p->h_xStop[s] - p->h_xStart[s]);
        sd[s] = make_int2(p->h_nDiasPtr[s], p->h_nDiasPtr[s + 1]);
        if (sd[s].y <= sd[s].x) return fail(TC_ERR_FORMAT, "shape %d has no diagonals", s);
        for (int n = sd[s].x + 1; n < sd[s].y; ++n)
            if (p->h_offsets[n] <= p->h_offsets[n - 1])
                return fail(TC_ERR_FORMAT, "offsets of shape %d are not increasing", s);
        p->max_span = std::max(p->max_span, p->h_offsets[sd[s].y - 1] - p->h_offsets[sd[s].x]);
    }
    for (Tile &t : tiles) t.nrows_kind |= diag_class(p, t.row0, t.row0 + tile_nrows(t)) << kDiagShift;

    // window plan: a second tile list for the window kernel (the batch and
    // served launches keep running `tiles`, with the same terms and order)
    std::vector<Tile> wtiles;
    p->nwtiles = 0;
    {
        int wlo = 0, whi = 0, wrows = 0, wnnz = 0;
        if (plan_window(p, csrRow, csrCol, wtiles, &wlo, &whi, &wrows, &wnnz)) {
            const int w_rp = (wrows + 8 + 3) & ~3, w_cw = (wnnz + 8 + 3) & ~3;
            const int w_xw = (wrows + whi - wlo + 8 + 3) & ~3;
            const size_t stage = 4 * (size_t)(w_rp + w_cw + w_xw);
            const int S = (int)std::min<size_t>(kWinMaxStages, (kWinSmemBudget - 128) / stage);
            if (S >= 2) {
                p->nwtiles = (int)wtiles.size();
                p->wlo = wlo;
                p->whi = whi;
                p->w_rp = w_rp;
                p->w_cw = w_cw;
                p->w_xw = w_xw;
                p->w_stages = S;
                p->w_grid = std::min(p->nwtiles, num_sms());
                for (Tile &t : wtiles) t.nrows_kind |= diag_class(p, t.row0, t.row0 + tile_nrows(t)) << kDiagShift;
            } else {
                wtiles.clear();
            }
        }
    }

    size_t o_rp = 0;
    size_t o_cols = align256(o_rp + sizeof(int) * ((size_t)M + 1) + 16);
    size_t o_tiles = align256(o_cols + sizeof(int) * (size_t)p->nnz_csr + 16);
    size_t o_sh = align256(o_tiles + sizeof(Tile) * tiles.size());
    size_t o_sd = align256(o_sh + sizeof(int4) * shapes.size());
    size_t o_off = align256(o_sd + sizeof(int2) * sd.size());
    size_t o_err = align256(o_off + sizeof(int) * (size_t)p->num_negs + 16);
    size_t o_wt = align256(o_err + 16);
    size_t total = align256(o_wt + sizeof(Tile) * wtiles.size());
    char *base = nullptr;
    cudaError_t e = cudaMalloc(&base, total);
    if (e != cudaSuccess)
        return fail(TC_ERR_ALLOC, "cudaMalloc(%zu) for the plan: %s", total, cudaGetErrorString(e));
    p->dev = base;
    p->dev_bytes = total;
    p->d_rowptr = reinterpret_cast<int *>(base + o_rp);
    p->d_cols = reinterpret_cast<int *>(base + o_cols);
    p->d_tiles = reinterpret_cast<Tile *>(base + o_tiles);
    p->d_shapes = reinterpret_cast<int4 *>(base + o_sh);
    p->d_shape_dias = reinterpret_cast<int2 *>(base + o_sd);
    p->d_offsets = reinterpret_cast<int *>(base + o_off);
    p->d_err = reinterpret_cast<int *>(base + o_err);
    p->d_wtiles = p->nwtiles ? reinterpret_cast<Tile *>(base + o_wt) : nullptr;
    {   // persistent grid: CTAs per SM from occupancy at this stage size
        DevPlan tmp = p->dev_plan();
        const size_t smem = stream_smem_bytes(tmp);
        int per_sm = 0;
        TC_CHECK(ensure_smem((const void *)spmv_tiles_kernel<false>, smem));
        TC_CHECK(ensure_smem((const void *)spmv_tiles_kernel<true>, smem));
        TC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, spmv_tiles_kernel<true>, kBlock, smem));
        const int cps = std::max(1, std::min(per_sm, p->params.ctas_per_sm));
        p->grid = std::max(1, std::min(p->ntiles, cps * num_sms()));
    }
    TC_CUDA(cudaMemsetAsync(base, 0, total, stream));
    TC_CUDA(cudaMemcpyAsync(p->d_rowptr, csrRow, sizeof(int) * ((size_t)M + 1),
                            cudaMemcpyHostToDevice, stream));
    if (p->nnz_csr)
        TC_CUDA(cudaMemcpyAsync(p->d_cols, csrCol, sizeof(int) * (size_t)p->nnz_csr,
                                cudaMemcpyHostToDevice, stream));
    if (!tiles.empty())
        TC_CUDA(cudaMemcpyAsync(p->d_tiles, tiles.data(), sizeof(Tile) * tiles.size(),
                                cudaMemcpyHostToDevice, stream));
    if (p->nwtiles) {
        TC_CUDA(cudaMemcpyAsync(p->d_wtiles, wtiles.data(), sizeof(Tile) * wtiles.size(),
                                cudaMemcpyHostToDevice, stream));
        DevPlan dp = p->dev_plan();
        TC_CHECK(window_prepare(dp));
    }
    if (!shapes.empty()) {
        TC_CUDA(cudaMemcpyAsync(p->d_shapes, shapes.data(), sizeof(int4) * shapes.size(),
                                cudaMemcpyHostToDevice, stream));
        TC_CUDA(cudaMemcpyAsync(p->d_shape_dias, sd.data(), sizeof(int2) * sd.size(),
                                cudaMemcpyHostToDevice, stream));
        TC_CUDA(cudaMemcpyAsync(p->d_offsets, p->h_offsets.data(), sizeof(int) * p->num_negs,
                                cudaMemcpyHostToDevice, stream));
    }
    TC_CUDA(cudaStreamSynchronize(stream));   // host arrays may be freed after return
    return TC_OK;
}

}  // namespace tc
