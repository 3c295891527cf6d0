// tc_internal.h -- shared definitions of libtaichi_b200 (not installed).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "taichi_b200.h"

namespace tc {

// ---------------------------------------------------------------- errors
void set_error(const char *fmt, ...);
tc_status fail(tc_status s, const char *fmt, ...);

// On failure the runtime's last-error state is cleared too, so a failed call
// is reported once, by the entry point that made it.
#define TC_CUDA(call)                                                              \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            (void)cudaGetLastError();                                              \
            return ::tc::fail(TC_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__,     \
                              #call, cudaGetErrorString(e_));                      \
        }                                                                          \
    } while (0)

// Raises the dynamic shared-memory limit of `kernel` on the current device to
// at least `bytes` (never lowers it, so earlier launches stay valid).
tc_status ensure_smem(const void *kernel, size_t bytes);

// Range checks of a tc_params (partition constants and tile shape);
// TC_ERR_INVALID with a message naming the field.
tc_status check_params(const tc_params &p);

#define TC_CHECK(st)                                                               \
    do {                                                                           \
        tc_status s_ = (st);                                                       \
        if (s_ != TC_OK) return s_;                                                \
    } while (0)

// ------------------------------------------------------------- tile plan
// A multiply tile is a run of consecutive rows processed by one CTA.  Kinds
// TILE_L1..TILE_L32 give 1..32 lanes to each row; TILE_MERGE splits the
// tile's rows and entries evenly over the threads; TILE_STREAM gathers every
// entry's x term into shared memory with coalesced word loads, then sums each
// row there; TILE_LONG gives one row a whole CTA.
enum TileKind : int {
    TILE_L1 = 0, TILE_L2 = 1, TILE_L4 = 2, TILE_L8 = 3, TILE_L16 = 4, TILE_L32 = 5,
    TILE_LONG = 6,
    TILE_MERGE = 7,    // merge-path split of rows and entries over the CTA's threads
    TILE_STREAM = 8,   // entry-parallel gather, then row-parallel sums in shared memory
    TILE_STREAM4 = 9,  // the same with 4 consecutive rows per thread (row0 % 4 == 0)
    TILE_DIRECT4 = 10,    // 4 consecutive rows per thread straight from global memory
    TILE_DIRECT_WIDE = 11, // the same over up to 4096 rows (a 1024-thread CTA)
    TILE_WINDOW = 12      // rows summed from a staged x window (the window kernel's tiles)
};

struct Tile {          // 16 bytes, read once per CTA
    int row0;          // first row
    int nz0;           // first CSR entry (rowptr[row0])
    int nnz;           // CSR entries of the tile
    int nrows_kind;    // nrows (bits 0-12) | diagonal class << 13 (15 bits) | kind << 28
};

// Diagonal class of a tile: how its rows meet the dense-diagonal shapes.
constexpr int kDiagGeneral = 0;        // per-row search over the shapes
constexpr int kDiagNone = 0x7fff;      // no row of the tile is in any shape
// otherwise s + 1: every row lies in shape s alone and every offset of s
// lands inside the shape's columns for every row of the tile
constexpr int kMaxTileNrows = 0x1fff;
constexpr int kDiagShift = 13;

__host__ __device__ inline int tile_nrows(const Tile &t) { return t.nrows_kind & 0x1fff; }
__host__ __device__ inline int tile_dclass(const Tile &t) { return (t.nrows_kind >> kDiagShift) & 0x7fff; }
__host__ __device__ inline int tile_kind(const Tile &t) { return (t.nrows_kind >> 28) & 0xf; }
__host__ __device__ inline int tile_word(int nrows, int kind) { return nrows | (kind << 28); }

constexpr int kBlock = 256;           // threads per CTA of the multiply kernels
constexpr int kMaxTileRows = 1 << 20; // planner limit on rows per tile
constexpr int kStageNnz = 8192;       // CSR words of a tile staged in shared memory
constexpr int kStreamNnz = 4096;      // most entries of a TILE_STREAM tile
constexpr int kStreamRows = 256;      // most rows of a TILE_STREAM tile (1 per thread)
constexpr int kStreamRowMax = 128;    // longer rows leave stream tiles for lane tiles
constexpr int kStream4Rows = 1024;    // most rows of a TILE_STREAM4 tile (a run of 4 per thread)
constexpr int kDirectRows = 1024;     // most rows of a direct tile (TILE_DIRECT4)
constexpr int kDirectWideBlock = 1024; // threads of the direct kernel's CTAs
constexpr int kPlanDiags = 8;         // dense diagonals a plan can carry in its launch parameters
// The rows kernel by default: stream plans whose rows average at most this
// many CSR words.  Measured per multiply against stream tiles: mesh (6.1
// words, hybrid) 39.4 against 45.7 µs; banded plain matrices of 9 words
// 12.6 / 12.7 µs, of 11 words 81.4 / 71.5 µs, of 12 words 5.4 / 5.1 µs.
constexpr int kRowsMeanMax = 8;
constexpr bool kRowsByDefault = true;
constexpr int kDirectWideRows = 4 * kDirectWideBlock;   // most rows of a TILE_DIRECT_WIDE tile
// A wide plan of at most kWideBoundTiles whole tiles passes each tile's
// first CSR word in the launch parameters (WideBounds), so a CTA loads its
// tile's words into shared memory (kWideWordQ int4s at most) at the same
// time as its row pointers instead of after them.
constexpr int kWideBoundTiles = 1024;
constexpr int kWideWordQ = 2048;
struct WideBounds {
    int nz[kWideBoundTiles + 1];
};
// A wide plan of at most kWideParamTiles tiles passes each tile's first CSR
// word in the launch parameters (2 KB), so a CTA prefetches its tile's words
// into L2 as it starts.
constexpr int kWideParamTiles = 511;
struct WideStarts {
    int nz[kWideParamTiles + 1];
};

// Window plans (tc_window.cu): tiles of consecutive rows whose row pointers,
// CSR words and x window are staged in shared memory by bulk copies.
constexpr int kWinBlock = 1024;       // threads of the window kernel's CTAs (one per SM)
constexpr int kWinRows = 1024;        // most rows of a window tile
constexpr int kWinNnz = 8192;         // most CSR words of a window tile
constexpr int kWinHalo = 4096;        // farthest column - row a window reaches, each side
constexpr int kWinMaxStages = 4;      // pipeline depth (stages of one CTA)
constexpr int kWinSmemBudget = 200 * 1024;   // shared memory of the stages
constexpr double kWinCover = 0.95;    // share of the in-halo accesses the window range holds

// Everything a multiply kernel needs about one plan (passed by value).
struct DevPlan {
    const int *rowptr;      // M+1
    const int *cols;        // nnz_csr (signed (col<<1|add) when hybrid)
    const Tile *tiles;      // ntiles
    const int4 *shapes;     // dia_shapes: {xStart, xStop, yStart, Msub}
    const int2 *shape_dias; // dia_shapes: {first offset, end offset}
    const int *offsets;     // num_negs
    int M, N, ntiles, dia_shapes, row_start, row_stop, hybrid;
    int max_span;           // widest offset span of any shape (max-min)
    int pdl;                // launch with programmatic stream serialization
    int stage_rp, stage_cw; // ints per shared-memory stage (row pointers, CSR words)
    int grid;               // persistent grid size
    int per_tile;           // one CTA per tile (stream plans): 1, or 2 when only stream,
                            // direct and long tiles occur (the lean kernel), 3 when
                            // every tile is a wide direct tile (the direct kernel), or 4
                            // when every tile is a stream tile (the stream kernel)
    int *err;               // device error word (1: a bounded wait gave up)
    int wide_rows;          // rows of each wide direct tile (the last may have fewer)
    // plans whose dense part is one shape of at most kPlanDiags offsets
    // (dn of them, in offset order): offset i adds x[r + d_col[i]] to the rows
    // r of [d_lo[i], d_hi[i]) and no other row has a diagonal term.  dn = 0:
    // no dense part, or more than one shape / more offsets (dgen = 1: the
    // per-row shape search, diag_row)
    int dn, dgen;
    int d_lo[kPlanDiags], d_hi[kPlanDiags], d_col[kPlanDiags];
    int rows;               // stream plan run by the rows kernel (one row per thread)
    int rows_w;             // the rows kernel's words loaded together (4, 6 or 8: from the usual row length)
    int pos;                // hybrid plan whose words are all additions (no holes)
    int ahead;              // stream / rows kernels: CTA b prefetches the operands of CTA b + ahead
    int prefetch;           // wide kernel: each CTA prefetches its tile's CSR words into L2
    int skew;               // stream tiles use skewed shared-memory slots (vslot)
    // window plan (nwtiles > 0): the multiply runs the window kernel over wtiles
    const Tile *wtiles;
    int nwtiles;
    int wlo, whi;           // x window of rows [r0, r0 + n): [r0 + wlo, r0 + n + whi)
    int w_rp, w_cw, w_xw;   // ints per stage: row pointers, CSR words, x window
    int w_stages, w_grid;   // pipeline depth, persistent grid
};

struct tc_plan_impl;

}  // namespace tc

// Opaque plan (the public tc_plan).
struct tc_plan {
    int M = 0, N = 0;
    tc_params params{};
    // format scalars (TaiChi_new)
    int dia_shapes = 0, num_negs = 0, dense_nnz = 0, zero_elements = 0, sparse_nnz = 0;
    int row_start = 0, row_stop = 0;
    int64_t nnz_input = 0, nnz_csr = 0;
    int hybrid = 0;
    // device arrays (one allocation, `dev`)
    void *dev = nullptr;
    size_t dev_bytes = 0;
    int *d_rowptr = nullptr, *d_cols = nullptr, *d_offsets = nullptr;
    tc::Tile *d_tiles = nullptr;
    int4 *d_shapes = nullptr;
    int2 *d_shape_dias = nullptr;
    int ntiles = 0, ntiles_vector = 0, ntiles_long = 0;
    int ntiles_lanes = 0;                // lane and merge tiles (TILE_L1..L32, TILE_MERGE)
    int ntiles_wide = 0;                 // TILE_DIRECT_WIDE tiles (all or none)
    int ntiles_stream = 0;               // TILE_STREAM tiles
    int max_span = 0;
    int stage_rp = 8, stage_cw = 8, grid = 1;
    int *d_err = nullptr;
    int wide_rows = 0;                   // rows of each wide direct tile
    int stream_skew = 0;                 // the plan's usual row length is a multiple of 8
    int rows_w = 8;                      // the rows kernel's words in flight (the usual row length, 4 / 6 / 8)
    int all_pos = 0;                     // hybrid plan with no holes (every word an addition)
    // window plan (tc_window.cu); nwtiles == 0 when the plan has none
    tc::Tile *d_wtiles = nullptr;
    int nwtiles = 0, wlo = 0, whi = 0, w_rp = 0, w_cw = 0, w_xw = 0, w_stages = 0, w_grid = 0;
    // host copies of the small format arrays (always) and optionally the CSR
    std::vector<int> h_xStart, h_yStart, h_xStop, h_nDiasPtr, h_offsets;
    std::vector<int> h_rowptr, h_cols;   // only with TC_FLAG_KEEP_HOST
    std::vector<int> h_wide_nz;          // wide plans: first CSR word of each tile, and the end
    std::vector<int> h_wide_z;           // the same for the word prefetch (WideStarts)
    // partition diagnostics
    double partition_ms = 0.0;
    int thumb_W = 0, thumb_H = 0;
    std::vector<unsigned char> thumb_stages;   // 5*H*W when kept
    std::vector<int> corners;                   // 4 per kept contour
    // device staging for tc_spmv_host
    // host-vector staging slots (tc_spmv_host: slot 0; tc_spmv_host_async:
    // any of TC_HOST_SLOTS)
    float *d_xbuf[TC_HOST_SLOTS] = {}, *d_ybuf[TC_HOST_SLOTS] = {};

    tc::DevPlan dev_plan() const;
    int64_t spmv_bytes() const;
};

namespace tc {
// Builds the tiles + device format from host arrays of an already formatted
// matrix (csrRow has M+1 entries).  Shared by every plan constructor.
tc_status plan_upload(tc_plan *p, const int *csrRow, const int *csrCol,
                      cudaStream_t stream);
// Host tile planner (row-length histogram -> tile kinds).
// Stream tiles hold at most nnz_csr / min_tiles entries (not below 512), so
// a small matrix still spreads over the GPU.
void plan_tiles(const int *rowptr, int M, const tc_params &prm, int min_tiles,
                std::vector<Tile> &tiles, int *nvec, int *nlong);
// Rows of a wide direct tile: the multiple of 4 that makes two equal tiles
// per SM (between kDirectRows and kDirectWideRows), so no SM holds twice the
// rows of another
// (R-MAT scale 20: 296 tiles of 3,544 rows; 4.99 against 5.20 us per
// multiply for 256 tiles of 4,096 rows on the same box); kDirectWideRows
// with TC_FLAG_WIDE_FIXED.
int wide_tile_rows(int M, const tc_params &prm, int sms);
// Resident CTAs per SM the lean one-CTA-per-tile kernel is compiled for
// (40 registers: the stream tiles' words, terms and row pointers fit
// without spills).
constexpr int kLeanMinBlocks = 6, kLeanMinBlocksSigned = 6;
// The stream-only kernel for plans of more tiles than one wave at that
// occupancy: 8 CTAs per SM at 32 registers (no spills).  Many waves of tiles
// gain from the extra resident loads (9-point mesh on 2048^2: 63.2 -> 52.5
// µs); a single wave loses from the thinner threads (n = 65,536 random
// matrix: 5.6 -> 6.7 µs), so a plan takes it only above one wave.
constexpr int kStreamManyMinBlocks = 8;
// The rows kernel: 8 CTAs per SM (32 registers) with one strip of rows per
// CTA, 4 with two.
constexpr int kRowsMinBlocks = 8;
// The same for the batch and served kernels, which read the plan descriptor
// from memory instead of the parameter bank (48 registers).
constexpr int kItemMinBlocks = 5;
// Launch of the multiply kernel for one plan.
// wb: the tiles' word bounds of a wide plan (nullptr: the kernels that read
// them from the tile list).  launch_plan passes the plan's own.
tc_status launch_spmv(const DevPlan &dp, const float *x, float *y, cudaStream_t s,
                      const WideBounds *wb = nullptr, const WideStarts *ws = nullptr);
tc_status launch_plan(const tc_plan *p, const float *x, float *y, cudaStream_t s);
// Window plans (tc_window.cu): the planner (false when the matrix does not
// qualify), the kernels' shared-memory setup and the launch.
bool plan_window(const tc_plan *p, const int *rowptr, const int *cols, std::vector<Tile> &wtiles, int *wlo,
                 int *whi, int *max_rows, int *max_nnz);
size_t window_smem_bytes(const DevPlan &dp);
tc_status window_prepare(DevPlan &dp);
tc_status launch_window(const DevPlan &dp, const float *x, float *y, cudaStream_t s);
tc_status launch_spmm(const DevPlan &dp, const float *X, int ldx, int k, float *Y, int ldy,
                      cudaStream_t s);

// GPU partitioner: device CSR in, format (host vectors) out.
struct PartitionOut {
    int dia_shapes = 0, num_negs = 0, dense_nnz = 0, zero_elements = 0, sparse_nnz = 0;
    int row_start = 0, row_stop = 0;
    std::vector<int> xStart, yStart, xStop, nDiasPtr, offsets;
    // device CSR remainder (allocated here with cudaMalloc; caller frees)
    int *d_rowptr = nullptr, *d_cols = nullptr;
    int64_t nnz_csr = 0;
    bool aliases_input = false;      // dense_nnz == 0: the input CSR is the format
    int thumb_W = 0, thumb_H = 0, ncontours = 0;
    std::vector<int> corners;
    std::vector<unsigned char> stages;
    std::vector<unsigned char> claimed;   // per input entry, when requested
    double ms = 0.0;
};
tc_status gpu_partition(int M, int N, int64_t nnz, const int *d_rowptr, const int *d_col,
                        const float *d_val, const tc_params &prm, bool keep_stages,
                        bool want_claimed, cudaStream_t s, PartitionOut &out);

// Matrix Market entries in file order (1-based indices, checked against the
// size line; symmetric / hermitian files flagged, not yet mirrored).
struct MtxEntry {
    int i, j;
    float v;
};
struct MtxCoo {
    int M = 0, N = 0;
    bool symmetric = false;
    std::vector<MtxEntry> entries;
};
// Parses a Matrix Market coordinate file (readMtx's grammar); *ref_code gets
// the reference's code (0, -1 open, -2 banner, -3 complex, -4 size, -5 entry).
tc_status mtx_parse(const char *path, MtxCoo &out, int *ref_code);

// Dense-diagonal extraction of one shape box on host arrays (marks h_val).
struct OneShape {
    int width = 0, neg = 0;
    long nnz = 0;
    std::vector<int> offs, start, end, nzero;
    std::vector<std::vector<int>> holes;   // local hole rows per dense diagonal
};
tc_status gpu_one_shape(int M, int64_t nnz, const int *h_rowptr, const int *h_col, float *h_val,
                        int x, int y, int a, int b, double density, OneShape &o);
}  // namespace tc
