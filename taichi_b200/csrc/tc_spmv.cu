// tc_spmv.cu -- the multiply: tile planner, device format upload and the
// value-free hybrid SpMV / SpMM kernels for sm_100a.
//
// Replaces taichi_SpMV's dispatch and kernels (TaiChi.cu:965-1329): the
// reference picks one of four CSR-vector kernels with a fixed vector width per
// matrix; here one kernel walks a precomputed list of row tiles whose kind
// (thread per row / warp per row / CTA per long row) was chosen from the
// row-length histogram, stages each tile's row pointers and CSR entries in
// shared memory with batched coalesced loads, streams the x window of every
// dense diagonal through shared memory with 16-byte loads, and writes y once
// (the diagonal and CSR parts are merged in registers).
//
// Arithmetic (per row, FP32): the signed CSR entries in stored order (holes
// subtract, leftovers add), then the dense diagonals shape by shape in offset
// order -- the same terms as TaiChi.cu:1007-1024.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "tc_internal.h"
#include "tc_tile.cuh"

namespace tc {

// ------------------------------------------------------------------ planner
void plan_tiles(const int *rp, int M, const tc_params &prm, std::vector<Tile> &tiles, int *nvec,
                int *nlong)
{
    const int rows_cap = std::max(1, std::min(prm.tile_rows, kMaxTileRows));
    const int nnz_cap = std::max(1, std::min(prm.tile_nnz, kMaxTileNnz));
    const int vthr = prm.vector_threshold;
    tiles.clear();
    *nvec = *nlong = 0;
    int r = 0;
    while (r < M) {
        int len = rp[r + 1] - rp[r];
        if (len > nnz_cap) {
            tiles.push_back(Tile{r, rp[r], len, 1 | (TILE_LONG << 28)});
            ++*nlong;
            ++r;
            continue;
        }
        int start = r, nnz = 0, maxlen = 0;
        while (r < M && r - start < rows_cap) {
            len = rp[r + 1] - rp[r];
            if (len > nnz_cap || nnz + len > nnz_cap) break;
            nnz += len;
            maxlen = std::max(maxlen, len);
            ++r;
        }
        int kind = maxlen > vthr ? TILE_VECTOR : TILE_SCALAR;
        *nvec += kind == TILE_VECTOR;
        tiles.push_back(Tile{start, rp[start], nnz, (r - start) | (kind << 28)});
    }
}

size_t spmv_smem_bytes(int rows_cap, int nnz_cap, int max_span)
{
    return spmv_smem_bytes_impl(rows_cap, nnz_cap, max_span);
}

// ------------------------------------------------------------------ kernels
namespace {

template <bool SIGNED>
__global__ void __launch_bounds__(kBlock) spmv_tiles_kernel(DevPlan p, const float *__restrict__ x,
                                                            float *__restrict__ y)
{
    extern __shared__ __align__(16) char smem[];
    for (int t = blockIdx.x; t < p.ntiles; t += gridDim.x) {
        const Tile tile = p.tiles[t];
        run_tile<SIGNED>(p, tile, x, y, smem);
        __syncthreads();
    }
}

// SpMM: one warp per row, lane l owns columns [l*V, l*V+V) of the k
// right-hand sides.
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
    for (int r = warp; r < p.M; r += nwarps) {
        float acc[V];
#pragma unroll
        for (int v = 0; v < V; ++v) acc[v] = 0.f;
        const int b = __ldg(p.rowptr + r), e = __ldg(p.rowptr + r + 1);
        for (int j0 = b; j0 < e; j0 += 32) {
            const int cnt = min(32, e - j0);
            const int mine = lane < cnt ? __ldg(p.cols + j0 + lane) : 0;
            for (int q = 0; q < cnt; ++q) {
                const int cv = __shfl_sync(0xffffffffu, mine, q);
                const int col = SIGNED ? (cv >> 1) : cv;
                const float sg = (!SIGNED || (cv & 1)) ? 1.f : -1.f;
                if (active) {
                    const float *xr = X + (size_t)col * ldx + c0;
#pragma unroll
                    for (int v = 0; v < V; ++v)
                        if (c0 + v < k) acc[v] += sg * __ldg(xr + v);
                }
            }
        }
        if (p.dia_shapes > 0 && r >= p.row_start && r < p.row_stop) {
            for (int s = 0; s < p.dia_shapes; ++s) {
                const int4 sh = __ldg(p.shapes + s);
                if (r < sh.x || r >= sh.y) continue;
                const int2 dr = __ldg(p.shape_dias + s);
                for (int n = dr.x; n < dr.y; ++n) {
                    const int col = r - sh.x + sh.z + __ldg(p.offsets + n);
                    if (col < sh.z || col >= sh.z + sh.w) continue;
                    if (active) {
                        const float *xr = X + (size_t)col * ldx + c0;
#pragma unroll
                        for (int v = 0; v < V; ++v)
                            if (c0 + v < k) acc[v] += __ldg(xr + v);
                    }
                }
            }
        }
        if (active) {
            float *yr = Y + (size_t)r * ldy + c0;
#pragma unroll
            for (int v = 0; v < V; ++v)
                if (c0 + v < k) yr[v] = acc[v];
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

template <bool SIGNED>
static tc_status launch_tiles(const DevPlan &dp, const float *x, float *y, cudaStream_t s)
{
    const size_t smem = spmv_smem_bytes(dp.rows_cap, dp.nnz_cap, dp.max_span);
    // Opt-in above 48 KB of dynamic shared memory, once per device and size.
    static size_t configured[2][64] = {};
    int dev = 0;
    TC_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(TC_ERR_UNSUPPORTED, "device index %d", dev);
    if (configured[SIGNED][dev] < smem) {
        TC_CUDA(cudaFuncSetAttribute(spmv_tiles_kernel<SIGNED>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured[SIGNED][dev] = smem;
    }
    int grid = dp.ntiles;
    if (grid <= 0) return TC_OK;
    spmv_tiles_kernel<SIGNED><<<grid, kBlock, smem, s>>>(dp, x, y);
    TC_CUDA(cudaGetLastError());
    return TC_OK;
}

tc_status launch_spmv(const DevPlan &dp, const float *x, float *y, cudaStream_t s)
{
    if (dp.M == 0) return TC_OK;
    return dp.hybrid ? launch_tiles<true>(dp, x, y, s) : launch_tiles<false>(dp, x, y, s);
}

tc_status launch_spmm(const DevPlan &dp, const float *X, int ldx, int k, float *Y, int ldy,
                      cudaStream_t s)
{
    if (dp.M == 0) return TC_OK;
    const int warps_needed = dp.M;
    int grid = std::min((warps_needed + kBlock / 32 - 1) / (kBlock / 32), num_sms() * 8);
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
    d.rows_cap = std::max(1, std::min(params.tile_rows, tc::kMaxTileRows));
    d.nnz_cap = std::max(1, std::min(params.tile_nnz, tc::kMaxTileNnz));
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

tc_status plan_upload(tc_plan *p, const int *csrRow, const int *csrCol, cudaStream_t stream)
{
    const int M = p->M;
    std::vector<Tile> tiles;
    plan_tiles(csrRow, M, p->params, tiles, &p->ntiles_vector, &p->ntiles_long);
    p->ntiles = (int)tiles.size();
    p->nnz_csr = csrRow[M];

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
    if (p->max_span > 8192) return fail(TC_ERR_UNSUPPORTED, "diagonal span %d too wide", p->max_span);

    size_t o_rp = 0;
    size_t o_cols = align256(o_rp + sizeof(int) * ((size_t)M + 1) + 16);
    size_t o_tiles = align256(o_cols + sizeof(int) * (size_t)p->nnz_csr + 16);
    size_t o_sh = align256(o_tiles + sizeof(Tile) * tiles.size());
    size_t o_sd = align256(o_sh + sizeof(int4) * shapes.size());
    size_t o_off = align256(o_sd + sizeof(int2) * sd.size());
    size_t total = align256(o_off + sizeof(int) * (size_t)p->num_negs + 16);
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
    TC_CUDA(cudaMemsetAsync(base, 0, total, stream));
    TC_CUDA(cudaMemcpyAsync(p->d_rowptr, csrRow, sizeof(int) * ((size_t)M + 1),
                            cudaMemcpyHostToDevice, stream));
    if (p->nnz_csr)
        TC_CUDA(cudaMemcpyAsync(p->d_cols, csrCol, sizeof(int) * (size_t)p->nnz_csr,
                                cudaMemcpyHostToDevice, stream));
    if (!tiles.empty())
        TC_CUDA(cudaMemcpyAsync(p->d_tiles, tiles.data(), sizeof(Tile) * tiles.size(),
                                cudaMemcpyHostToDevice, stream));
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
