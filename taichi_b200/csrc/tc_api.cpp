// tc_api.cpp -- the extern "C" entry points of libtaichi_b200 (taichi_b200.h).

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstring>
#include <new>

#include "tc_internal.h"

namespace tc {

static thread_local char g_err[1024] = "";

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

tc_status fail(tc_status s, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return s;
}

}  // namespace tc

using tc::fail;

extern "C" {

const char *tc_last_error(void) { return tc::g_err; }

const char *tc_status_string(tc_status s)
{
    switch (s) {
    case TC_OK: return "ok";
    case TC_ERR_INVALID: return "invalid argument";
    case TC_ERR_CUDA: return "CUDA error";
    case TC_ERR_ALLOC: return "allocation failed";
    case TC_ERR_IO: return "I/O or parse error";
    case TC_ERR_FORMAT: return "inconsistent format";
    case TC_ERR_CAPACITY: return "capacity exceeded";
    case TC_ERR_TIMEOUT: return "device wait timed out";
    case TC_ERR_UNSUPPORTED: return "unsupported";
    }
    return "unknown status";
}

void tc_params_default(tc_params *p)
{
    if (!p) return;
    p->thumb_height = 512;     // morohutils.cu:191
    p->open_len = 30;          // morohutils.cu:239,242
    p->eye_size = 5;           // morohutils.cu:250
    p->min_contour = 80;       // morohutils.cu:140
    p->min_shape_side = 1000;  // TaiChi.cu:379
    p->density = 0.6;          // TaiChi.cu:757
    p->tile_rows = 1024;
    p->tile_nnz = 2048;
    p->max_lanes = 32;
    p->ctas_per_sm = 4;
    p->tile_mode = 2;
    p->flags = 0;
    p->rows_w = 0;
}

}  // extern "C"

tc_status tc::check_params(const tc_params &p)
{
    if (p.thumb_height < 2 || p.thumb_height > 4096)
        return fail(TC_ERR_INVALID, "thumb_height %d outside [2, 4096]", p.thumb_height);
    if (p.open_len < 1 || p.open_len > 256 || p.eye_size < 1 || p.eye_size > 63)
        return fail(TC_ERR_INVALID, "morphology element sizes out of range");
    if (p.tile_rows < 1 || p.tile_rows > tc::kMaxTileRows)
        return fail(TC_ERR_INVALID, "tile_rows %d outside [1, %d]", p.tile_rows, tc::kMaxTileRows);
    if (p.tile_nnz < 1) return fail(TC_ERR_INVALID, "tile_nnz %d < 1", p.tile_nnz);
    if (p.tile_mode < 0 || p.tile_mode > 2)
        return fail(TC_ERR_INVALID, "tile_mode %d is not 0, 1 or 2", p.tile_mode);
    if (p.ctas_per_sm < 1 || p.ctas_per_sm > 32)
        return fail(TC_ERR_INVALID, "ctas_per_sm %d outside [1, 32]", p.ctas_per_sm);
    if (p.max_lanes < 1 || p.max_lanes > 32 || (p.max_lanes & (p.max_lanes - 1)))
        return fail(TC_ERR_INVALID, "max_lanes %d is not a power of two in [1, 32]", p.max_lanes);
    if (p.rows_w != 0 && p.rows_w != 4 && p.rows_w != 6 && p.rows_w != 8)
        return fail(TC_ERR_INVALID, "rows_w %d is not 0, 4, 6 or 8", p.rows_w);
    return TC_OK;
}

using tc::check_params;

extern "C" {

// Validates a host format and builds a plan from it.
tc_status tc_plan_from_format(int M, int N, const tc_format *f, const tc_params *params,
                              void *stream, tc_plan **out)
{
    if (!f || !out || M < 0 || N < 0) return fail(TC_ERR_INVALID, "tc_plan_from_format: bad arguments");
    *out = nullptr;
    tc_params prm;
    tc_params_default(&prm);
    if (params) prm = *params;
    TC_CHECK(check_params(prm));
    if (f->dia_shapes < 0 || f->num_negs < 0) return fail(TC_ERR_FORMAT, "negative counts");
    if (f->dia_shapes > 0 && (!f->xStart || !f->yStart || !f->xStop || !f->nDiasPtr || !f->neg_offsets))
        return fail(TC_ERR_FORMAT, "shape arrays missing");
    if (M > 0 && !f->csrRow && !(f->dia_shapes > 0 && f->zero_elements + f->sparse_nnz == 0))
        return fail(TC_ERR_FORMAT, "csrRow missing");
    const bool hybrid = f->dia_shapes > 0;
    if (hybrid && N >= (1 << 30)) return fail(TC_ERR_UNSUPPORTED, "N >= 2^30 with signed columns");

    tc_plan *p = new (std::nothrow) tc_plan();
    if (!p) return fail(TC_ERR_ALLOC, "host allocation");
    p->M = M; p->N = N; p->params = prm;
    p->dia_shapes = f->dia_shapes; p->num_negs = f->num_negs; p->dense_nnz = f->dense_nnz;
    p->zero_elements = f->zero_elements; p->sparse_nnz = f->sparse_nnz;
    p->row_start = f->row_start; p->row_stop = f->row_stop;
    p->hybrid = hybrid;
    if (hybrid) {
        p->h_xStart.assign(f->xStart, f->xStart + f->dia_shapes);
        p->h_yStart.assign(f->yStart, f->yStart + f->dia_shapes);
        p->h_xStop.assign(f->xStop, f->xStop + f->dia_shapes);
        p->h_nDiasPtr.assign(f->nDiasPtr, f->nDiasPtr + f->dia_shapes + 1);
        p->h_offsets.assign(f->neg_offsets, f->neg_offsets + f->num_negs);
        for (int s = 0; s < f->dia_shapes; ++s) {
            int xs = f->xStart[s], xe = f->xStop[s], ys = f->yStart[s];
            if (xs < 0 || xe > M || xs >= xe || ys < 0 || ys + (xe - xs) > N) {
                delete p;
                return fail(TC_ERR_FORMAT, "shape %d box [%d,%d) x [%d,+%d) outside %d x %d", s, xs,
                            xe, ys, xe - xs, M, N);
            }
        }
        if (f->nDiasPtr[0] != 0 || f->nDiasPtr[f->dia_shapes] != f->num_negs) {
            delete p;
            return fail(TC_ERR_FORMAT, "nDiasPtr does not span neg_offsets");
        }
        for (int s = 0; s < f->dia_shapes; ++s)
            if (f->nDiasPtr[s + 1] < f->nDiasPtr[s]) {
                delete p;
                return fail(TC_ERR_FORMAT, "nDiasPtr decreases at shape %d", s);
            }
    }
    std::vector<int> zero_rp;
    const int *rp = f->csrRow;
    if (!rp) { zero_rp.assign((size_t)M + 1, 0); rp = zero_rp.data(); }
    const int64_t nnz_csr = M > 0 ? rp[M] : 0;
    for (int r = 0; r < M; ++r)
        if (rp[r + 1] < rp[r]) { delete p; return fail(TC_ERR_FORMAT, "csrRow decreases at row %d", r); }
    if (rp[0] != 0) { delete p; return fail(TC_ERR_FORMAT, "csrRow[0] != 0"); }
    const int lim = hybrid ? 2 * N : N;
    for (int64_t j = 0; j < nnz_csr; ++j)
        if (f->csrCol[j] < 0 || f->csrCol[j] >= lim) {
            delete p;
            return fail(TC_ERR_FORMAT, "csrCol[%lld] = %d outside the matrix", (long long)j, f->csrCol[j]);
        }
    p->nnz_input = (int64_t)f->dense_nnz + f->sparse_nnz;
    if (prm.flags & TC_FLAG_KEEP_HOST) {
        p->h_rowptr.assign(rp, rp + M + 1);
        p->h_cols.assign(f->csrCol, f->csrCol + nnz_csr);
    }
    tc_status st = tc::plan_upload(p, rp, f->csrCol, (cudaStream_t)stream);
    if (st != TC_OK) { tc_plan_destroy(p); return st; }
    *out = p;
    return TC_OK;
}

tc_status tc_plan_destroy(tc_plan *p)
{
    if (!p) return TC_OK;
    if (p->dev) cudaFree(p->dev);
    for (int k = 0; k < TC_HOST_SLOTS; ++k) {
        if (p->d_xbuf[k]) cudaFree(p->d_xbuf[k]);
        if (p->d_ybuf[k]) cudaFree(p->d_ybuf[k]);
    }
    delete p;
    return TC_OK;
}

tc_status tc_plan_info_get(const tc_plan *p, tc_plan_info *i)
{
    if (!p || !i) return fail(TC_ERR_INVALID, "null argument");
    memset(i, 0, sizeof *i);
    i->M = p->M; i->N = p->N;
    i->dia_shapes = p->dia_shapes; i->num_negs = p->num_negs; i->dense_nnz = p->dense_nnz;
    i->zero_elements = p->zero_elements; i->sparse_nnz = p->sparse_nnz;
    i->row_start = p->row_start; i->row_stop = p->row_stop;
    i->nnz_input = p->nnz_input; i->nnz_csr = p->nnz_csr;
    i->ntiles = p->ntiles; i->ntiles_vector = p->ntiles_vector; i->ntiles_long = p->ntiles_long;
    i->device_bytes = (int64_t)p->dev_bytes;
    i->spmv_bytes = p->spmv_bytes();
    i->partition_ms = p->partition_ms;
    i->num_contours = (int)(p->corners.size() / 4);
    i->nwtiles = p->nwtiles;
    i->window_lo = p->wlo;
    i->window_hi = p->whi;
    {
        const tc::DevPlan d = p->dev_plan();
        i->kernel = d.nwtiles > 0 ? TC_KERNEL_WINDOW : d.per_tile == 4 && d.rows ? TC_KERNEL_ROWS
                  : d.per_tile == 0 ? TC_KERNEL_TILES : d.per_tile == 1 ? TC_KERNEL_GRID
                  : d.per_tile == 2 ? TC_KERNEL_LEAN : d.per_tile == 3 ? TC_KERNEL_WIDE : TC_KERNEL_STREAM;
    }
    return TC_OK;
}

tc_status tc_plan_export(const tc_plan *p, int *xStart, int *yStart, int *xStop, int *nDiasPtr,
                         int *neg_offsets, int *csrRow, int *csrCol)
{
    if (!p) return fail(TC_ERR_INVALID, "null plan");
    auto put = [](int *dst, const std::vector<int> &v) {
        if (dst && !v.empty()) memcpy(dst, v.data(), v.size() * sizeof(int));
    };
    put(xStart, p->h_xStart); put(yStart, p->h_yStart); put(xStop, p->h_xStop);
    put(nDiasPtr, p->h_nDiasPtr); put(neg_offsets, p->h_offsets);
    if (csrRow) TC_CUDA(cudaMemcpy(csrRow, p->d_rowptr, sizeof(int) * ((size_t)p->M + 1), cudaMemcpyDeviceToHost));
    if (csrCol && p->nnz_csr)
        TC_CUDA(cudaMemcpy(csrCol, p->d_cols, sizeof(int) * (size_t)p->nnz_csr, cudaMemcpyDeviceToHost));
    return TC_OK;
}

tc_status tc_plan_thumbnail(const tc_plan *p, unsigned char *stages, int *W, int *corners,
                            int *ncorners)
{
    if (!p) return fail(TC_ERR_INVALID, "null plan");
    if (W) *W = p->thumb_W;
    if (ncorners) *ncorners = (int)(p->corners.size() / 4);
    if (corners && !p->corners.empty()) memcpy(corners, p->corners.data(), p->corners.size() * sizeof(int));
    if (stages && !p->thumb_stages.empty()) memcpy(stages, p->thumb_stages.data(), p->thumb_stages.size());
    return TC_OK;
}

tc_status tc_plan_check(const tc_plan *p)
{
    if (!p) return fail(TC_ERR_INVALID, "null plan");
    int e = 0;
    TC_CUDA(cudaMemcpy(&e, p->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (!e) return TC_OK;
    TC_CUDA(cudaMemset(p->d_err, 0, sizeof(int)));   // reported once: the next multiply starts clean
    return fail(TC_ERR_TIMEOUT, "a multiply of this plan gave up waiting for its staged tiles");
}

tc_status tc_spmv(const tc_plan *p, const float *d_x, float *d_y, void *stream)
{
    if (!p || (!d_x && p->N) || (!d_y && p->M)) return fail(TC_ERR_INVALID, "tc_spmv: null argument");
    return tc::launch_plan(p, d_x, d_y, (cudaStream_t)stream);
}

// The device address through which a kernel may store into h_y, or null when
// h_y is not page-locked host memory mapped for the current device (pageable
// memory, device memory, or a registration without a device mapping).
static float *mapped_host_y(float *h_y)
{
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, h_y) != cudaSuccess) {
        cudaGetLastError();                  // an unknown pointer: not an error of this call
        return nullptr;
    }
    return a.type == cudaMemoryTypeHost ? static_cast<float *>(a.devicePointer) : nullptr;
}

// Copy x in, multiply, copy y out on `stream`, through the plan's staging
// slot `slot` (device x / y buffers allocated on first use).  With
// TC_FLAG_HOST_Y_MAPPED and a mapped page-locked h_y the multiply stores y
// into h_y itself (every kernel writes y with plain stores only) and there
// is no copy-out; a plan without columns keeps the copy (its y = 0 is a
// device memset).
static tc_status spmv_host_enqueue(tc_plan *p, const float *h_x, float *h_y, int slot, cudaStream_t s)
{
    float *yk = nullptr;
    if ((p->params.flags & TC_FLAG_HOST_Y_MAPPED) && p->M && p->N) yk = mapped_host_y(h_y);
    float *&dx = p->d_xbuf[slot];
    float *&dy = p->d_ybuf[slot];
    if (!dx) {
        cudaError_t e1 = cudaMalloc(&dx, sizeof(float) * ((size_t)p->N + 4));
        if (e1 != cudaSuccess) return fail(TC_ERR_ALLOC, "x staging buffer");
    }
    if (!dy && !yk) {
        cudaError_t e2 = cudaMalloc(&dy, sizeof(float) * ((size_t)p->M + 4));
        if (e2 != cudaSuccess) return fail(TC_ERR_ALLOC, "y staging buffer");
    }
    if (p->N) TC_CUDA(cudaMemcpyAsync(dx, h_x, sizeof(float) * (size_t)p->N, cudaMemcpyHostToDevice, s));
    if (yk) return tc::launch_plan(p, dx, yk, s);
    TC_CHECK(tc::launch_plan(p, dx, dy, s));
    if (p->M) TC_CUDA(cudaMemcpyAsync(h_y, dy, sizeof(float) * (size_t)p->M, cudaMemcpyDeviceToHost, s));
    return TC_OK;
}

tc_status tc_spmv_host(const tc_plan *cp, const float *h_x, float *h_y, void *stream)
{
    tc_plan *p = const_cast<tc_plan *>(cp);
    if (!p || (!h_x && p->N) || (!h_y && p->M)) return fail(TC_ERR_INVALID, "tc_spmv_host: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    TC_CHECK(spmv_host_enqueue(p, h_x, h_y, 0, s));
    TC_CUDA(cudaStreamSynchronize(s));
    return tc_plan_check(p);
}

tc_status tc_spmv_host_async(const tc_plan *cp, const float *h_x, float *h_y, int slot, void *stream)
{
    tc_plan *p = const_cast<tc_plan *>(cp);
    if (!p || (!h_x && p->N) || (!h_y && p->M) || slot < 0 || slot >= TC_HOST_SLOTS)
        return fail(TC_ERR_INVALID, "tc_spmv_host_async: null argument or slot outside [0, %d)", TC_HOST_SLOTS);
    return spmv_host_enqueue(p, h_x, h_y, slot, (cudaStream_t)stream);
}

tc_status tc_spmm(const tc_plan *p, const float *d_X, int ldx, int k, float *d_Y, int ldy, void *stream)
{
    if (!p || k < 1 || k > 64 || ldx < k || ldy < k) return fail(TC_ERR_INVALID, "tc_spmm: k must be in [1, 64], ld >= k");
    if ((!d_X && p->N) || (!d_Y && p->M)) return fail(TC_ERR_INVALID, "tc_spmm: null argument");
    return tc::launch_spmm(p->dev_plan(), d_X, ldx, k, d_Y, ldy, (cudaStream_t)stream);
}

// Builds a plan from a CSR pattern, partitioning it on the GPU unless
// TC_FLAG_NO_PARTITION is set.
tc_status tc_plan_create(int M, int N, int64_t nnz, const int *rowptr, const int *col,
                         const float *val, int on_device, const tc_params *params, void *stream,
                         tc_plan **out)
{
    if (!out || M < 0 || N < 0 || nnz < 0 || (M > 0 && !rowptr) || (nnz > 0 && !col))
        return fail(TC_ERR_INVALID, "tc_plan_create: bad arguments");
    if (nnz > INT32_MAX) return fail(TC_ERR_UNSUPPORTED, "more than 2^31-1 non-zeros");
    *out = nullptr;
    tc_params prm;
    tc_params_default(&prm);
    if (params) prm = *params;
    TC_CHECK(check_params(prm));
    cudaStream_t s = (cudaStream_t)stream;

    // host copies of the CSR (the planner needs row pointers on the host)
    std::vector<int> h_rp((size_t)M + 1), h_col;
    if (on_device) {
        TC_CUDA(cudaMemcpyAsync(h_rp.data(), rowptr, sizeof(int) * ((size_t)M + 1), cudaMemcpyDeviceToHost, s));
        TC_CUDA(cudaStreamSynchronize(s));
    } else {
        memcpy(h_rp.data(), rowptr, sizeof(int) * ((size_t)M + 1));
    }
    if (h_rp[0] != 0 || h_rp[M] != nnz) return fail(TC_ERR_FORMAT, "rowptr[0] != 0 or rowptr[M] != nnz");

    if (prm.flags & TC_FLAG_NO_PARTITION) {
        if (on_device) {
            h_col.resize((size_t)nnz);
            if (nnz) TC_CUDA(cudaMemcpy(h_col.data(), col, sizeof(int) * (size_t)nnz, cudaMemcpyDeviceToHost));
        }
        tc_format f{};
        f.sparse_nnz = (int)nnz;
        f.csrRow = h_rp.data();
        f.csrCol = on_device ? h_col.data() : col;
        return tc_plan_from_format(M, N, &f, &prm, stream, out);
    }

    // GPU partition from a device copy of the input
    int *d_rp = nullptr, *d_col = nullptr;
    float *d_val = nullptr;
    bool own = !on_device;
    if (own) {
        if (cudaMalloc(&d_rp, sizeof(int) * ((size_t)M + 1)) != cudaSuccess ||
            cudaMalloc(&d_col, sizeof(int) * (size_t)std::max<int64_t>(nnz, 1)) != cudaSuccess)
            return fail(TC_ERR_ALLOC, "device copy of the input CSR");
        TC_CUDA(cudaMemcpyAsync(d_rp, rowptr, sizeof(int) * ((size_t)M + 1), cudaMemcpyHostToDevice, s));
        if (nnz) TC_CUDA(cudaMemcpyAsync(d_col, col, sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice, s));
        if (val) {
            if (cudaMalloc(&d_val, sizeof(float) * (size_t)std::max<int64_t>(nnz, 1)) != cudaSuccess)
                return fail(TC_ERR_ALLOC, "device copy of the input values");
            if (nnz) TC_CUDA(cudaMemcpyAsync(d_val, val, sizeof(float) * (size_t)nnz, cudaMemcpyHostToDevice, s));
        }
    } else {
        d_rp = const_cast<int *>(rowptr);
        d_col = const_cast<int *>(col);
        d_val = const_cast<float *>(val);
    }
    tc::PartitionOut po;
    tc_status st = tc::gpu_partition(M, N, nnz, d_rp, d_col, d_val, prm,
                                     (prm.flags & TC_FLAG_KEEP_HOST) != 0, false, s, po);
    std::vector<int> fr, fc;
    if (st == TC_OK) {
        if (po.aliases_input) {
            fr = h_rp;
            if (on_device) {
                fc.resize((size_t)nnz);
                if (nnz) st = cudaMemcpy(fc.data(), col, sizeof(int) * (size_t)nnz, cudaMemcpyDeviceToHost) == cudaSuccess ? TC_OK : fail(TC_ERR_CUDA, "copy of the input columns");
            }
        } else {
            fr.resize((size_t)M + 1);
            fc.resize((size_t)po.nnz_csr);
            if (cudaMemcpy(fr.data(), po.d_rowptr, sizeof(int) * ((size_t)M + 1), cudaMemcpyDeviceToHost) != cudaSuccess ||
                (po.nnz_csr && cudaMemcpy(fc.data(), po.d_cols, sizeof(int) * (size_t)po.nnz_csr, cudaMemcpyDeviceToHost) != cudaSuccess))
                st = fail(TC_ERR_CUDA, "copy of the partitioned CSR");
        }
    }
    if (po.d_rowptr) cudaFree(po.d_rowptr);
    if (po.d_cols) cudaFree(po.d_cols);
    if (own) { cudaFree(d_rp); cudaFree(d_col); if (d_val) cudaFree(d_val); }
    if (st != TC_OK) return st;

    tc_format f{};
    f.dia_shapes = po.dia_shapes; f.num_negs = po.num_negs; f.dense_nnz = po.dense_nnz;
    f.zero_elements = po.zero_elements; f.sparse_nnz = po.sparse_nnz;
    f.row_start = po.row_start; f.row_stop = po.row_stop;
    f.xStart = po.xStart.data(); f.yStart = po.yStart.data(); f.xStop = po.xStop.data();
    f.nDiasPtr = po.nDiasPtr.data(); f.neg_offsets = po.offsets.data();
    f.csrRow = fr.data();
    f.csrCol = po.aliases_input && !on_device ? col : fc.data();
    tc_plan *p = nullptr;
    TC_CHECK(tc_plan_from_format(M, N, &f, &prm, stream, &p));
    p->nnz_input = nnz;
    p->partition_ms = po.ms;
    p->thumb_W = po.thumb_W;
    p->thumb_H = po.thumb_H;
    p->corners = po.corners;
    p->thumb_stages.swap(po.stages);
    *out = p;
    return TC_OK;
}

}  // extern "C"

#include <map>
#include <mutex>

namespace tc {

tc_status ensure_smem(const void *kernel, size_t bytes)
{
    // The default limit covers 48 KB of static + dynamic shared memory, so a
    // kernel with static shared memory may need the attribute for less than
    // 48 KB of dynamic memory too: set it for every size not yet granted.
    if (bytes == 0) return TC_OK;
    int dev = 0;
    TC_CUDA(cudaGetDevice(&dev));
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, size_t> done;
    std::lock_guard<std::mutex> lk(mu);
    size_t &v = done[{kernel, dev}];
    if (v >= bytes) return TC_OK;
    TC_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    v = bytes;
    return TC_OK;
}

}  // namespace tc
