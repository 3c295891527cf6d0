// tc_compat.cpp -- the reference's C++ entry points (TaiChi.h) served by the
// B200 library, so a program written against the reference links unchanged.
//
// Behaviour kept from the reference: return codes and messages of readMtx,
// the FLT_MAX marks that partition_shapes leaves in the caller's csrVal, the
// aliasing of the caller's CSR when no dense diagonal is found, the printed
// statistics and timings, and free_taichi_new freeing the struct itself.
// Deliberate differences: taichi_SpMV does not end with cudaDeviceReset()
// unless TAICHI_B200_DEVICE_RESET=1 (a reset would tear down every other
// library's CUDA state in the process), and a format whose CSR remainder is
// empty multiplies correctly (the reference reads an unallocated pointer).

#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>

#include "TaiChi.h"
#include "tc_internal.h"

namespace {

int env_int(const char *name, int dflt)
{
    const char *v = getenv(name);
    return v && *v ? atoi(v) : dflt;
}

double now_ms()
{
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

// TaiChi.cu:120-278
int readMtx(char *filename, int &m, int &n, unsigned long &nnzA, int *&csrRowPtrA,
            int *&csrColIdxA, float *&csrValA)
{
    int M = 0, N = 0, code = 0;
    int64_t nnz = 0;
    int *rp = nullptr, *ci = nullptr;
    float *va = nullptr;
    tc_status st = tc_read_mtx(filename, &M, &N, &nnz, &rp, &ci, &va, &code);
    if (st != TC_OK) {
        if (code == -2) printf("Could not process Matrix Market banner.\n");
        else if (code == -3) printf("Sorry, data type 'COMPLEX' is not supported. \n");
        else if (code == -5) printf("readMtx: %s\n", tc_last_error());
        return code ? code : -4;
    }
    m = M; n = N; nnzA = (unsigned long)nnz;
    csrRowPtrA = rp; csrColIdxA = ci; csrValA = va;
    return 0;
}

// TaiChi.cu:280-311
void cal_shape_size(int M, int N, int mF, int x1, int y1, int a1, int b1, int &x, int &y, int &a,
                    int &b, float &gain)
{
    if (M > mF) {
        gain = (float)M / (float)mF;
        x = (int)((float)x1 * gain); y = (int)((float)y1 * gain);
        a = (int)((float)a1 * gain); b = (int)((float)b1 * gain);
    } else if (M < mF) {
        gain = (float)mF / (float)M;
        x = (int)((float)x1 / gain); y = (int)((float)y1 / gain);
        a = (int)((float)a1 / gain); b = (int)((float)b1 / gain);
    } else {
        gain = 1.0f; x = x1; y = y1; a = a1; b = b1;
    }
    if (x < 0) x = 0;
    if (x > M - 1) x = M - 1;
    if (y < 0) y = 0;
    if (y > N - 1) y = N - 1;
    if (y + a > N) a = N - y;
    if (x + b > M) b = M - x;
    if (a > b) a = b; else b = a;
}

// TaiChi.cu:881-916
void cal_start_end(int M_sub, int N_sub, int width, int off, int n, int &start, int &end)
{
    const int ao = off < 0 ? -off : off;
    if (M_sub >= N_sub) {
        if (n >= width - 1) { start = 0; end = N_sub - off; }
        else if (ao > M_sub - N_sub) { start = ao; end = M_sub; }
        else { start = ao; end = N_sub + ao; }
    } else {
        if (n <= width - 1) { start = ao; end = M_sub; }
        else if (ao > N_sub - M_sub) { start = 0; end = N_sub - ao; }
        else { start = 0; end = M_sub; }
    }
}

// TaiChi.cu:947-963
int max(int *a, int len)
{
    int v = a[0];
    for (int i = 1; i < len; ++i) v = a[i] > v ? a[i] : v;
    return v;
}

int min(int *a, int len)
{
    int v = a[0];
    for (int i = 1; i < len; ++i) v = a[i] < v ? a[i] : v;
    return v;
}

// TaiChi.cu:918-945
void queryDevice()
{
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    printf("cudaError = %d\n", (int)e);
    for (int i = 0; i < count; ++i) {
        cudaDeviceProp p;
        cudaGetDeviceProperties(&p, i);
        printf("Device %d's main property: \n", i);
        printf("Device Name: %s\n", p.name);
        printf("Global Memory of device: %zu MB\n", p.totalGlobalMem / 1024 / 1024);
        printf("Maximal available shared memory for a block: %zu KB\n", p.sharedMemPerBlock / 1024);
        printf("Number of available registers for a block: %d\n", p.regsPerBlock);
        printf("Maximal number of threads for a block: %d\n", p.maxThreadsPerBlock);
        printf("Compute Capability: %d.%d\n", p.major, p.minor);
        printf("Number of multi processors: %d\n", p.multiProcessorCount);
    }
    if (cudaSetDevice(0) != cudaSuccess) printf("cudaSetDevice failed!");
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) printf("cudaGetDevice failed!");
    printf("\nThe device now beening used is device %d\n\n", dev);
}

// TaiChi.cu:77-118: frees the arrays and the struct; the CSR arrays are not
// freed when they alias the caller's input (dense_nnz == 0).
void free_taichi_new(TaiChi_new *t)
{
    if (!t) return;
    free(t->xStart); free(t->yStart); free(t->xStop); free(t->nDiasPtr); free(t->neg_offsets);
    if (t->dense_nnz > 0) { free(t->csrRow); free(t->csrCol); }
    free(t);
}

// TaiChi.cu:640-675
void free_taichi(int num_shapes, TaiChi *t)
{
    if (!t) return;
    for (int i = 0; i < num_shapes; ++i) {
        free(t[i].neg_offsets);
        free(t[i].numZeroNeg);
        if (t[i].rowZeroNeg)
            for (int d = 0; d < t[i].neg; ++d) free(t[i].rowZeroNeg[d]);
        free(t[i].rowZeroNeg);
        free(t[i].start); free(t[i].end); free(t[i].cStart);
    }
    free(t);
}

// TaiChi.cu:677-879: one shape box; the histogram, density test, hole rows
// and claims run on the GPU, the result fills the reference's TaiChi record
// (arrays malloc'd, released by free_taichi) and csrVal gets FLT_MAX marks.
void partition_dia_shape(int M, int N, int nnz, int *&csrRow, int *&csrCol, float *&csrVal,
                         float gain, shape &hi, TaiChi &t)
{
    (void)N; (void)gain;
    t.M_sub = hi.b; t.N_sub = hi.a; t.xStart = hi.x; t.yStart = hi.y;
    t.shape = 0;
    tc::OneShape o;
    tc_status st = tc::gpu_one_shape(M, nnz, csrRow, csrCol, csrVal, hi.x, hi.y, hi.a, hi.b, 0.6, o);
    if (st != TC_OK) {
        printf("CUDA Runtime Error: %s\n", tc_last_error());
        t.neg = 0;
        return;
    }
    t.width = o.width;
    t.neg = o.neg;
    if (o.neg <= 0) return;
    auto dup = [](const std::vector<int> &v) {
        int *p = (int *)malloc(std::max<size_t>(v.size(), 1) * sizeof(int));
        if (!v.empty()) memcpy(p, v.data(), v.size() * sizeof(int));
        return p;
    };
    t.neg_offsets = dup(o.offs);
    t.start = dup(o.start);
    t.end = dup(o.end);
    t.numZeroNeg = dup(o.nzero);
    t.cStart = (int *)malloc(sizeof(int) * o.neg);
    int maxz = 0;
    for (int d = 0; d < o.neg; ++d) {
        t.cStart[d] = o.offs[d] > 0 ? o.offs[d] : 0;
        maxz = std::max(maxz, o.nzero[d]);
    }
    t.nnz = (int)o.nnz;
    t.maxNumZero = maxz;
    t.rowZeroNeg = (int **)calloc(o.neg, sizeof(int *));
    if (maxz > 0)
        for (int d = 0; d < o.neg; ++d) {
            t.rowZeroNeg[d] = (int *)malloc(sizeof(int) * maxz);
            if (!o.holes[d].empty()) memcpy(t.rowZeroNeg[d], o.holes[d].data(), o.holes[d].size() * sizeof(int));
        }
}

// TaiChi.cu:313-638: the partition runs on the GPU; the result is returned
// in malloc'd host arrays exactly as the reference lays them out.
void partition_shapes(char *sdf_name, int M, int N, int nnz, int *&csrRow, int *&csrCol,
                      float *&csrVal, TaiChi_new *t)
{
    (void)sdf_name;
    tc_params prm;
    tc_params_default(&prm);
    int *d_rp = nullptr, *d_col = nullptr;
    float *d_val = nullptr;
    const size_t nz = (size_t)std::max(nnz, 0);
    if (cudaMalloc(&d_rp, sizeof(int) * ((size_t)M + 1)) != cudaSuccess ||
        cudaMalloc(&d_col, sizeof(int) * std::max<size_t>(nz, 1)) != cudaSuccess ||
        cudaMalloc(&d_val, sizeof(float) * std::max<size_t>(nz, 1)) != cudaSuccess) {
        printf("CUDA Runtime Error: %s\n", "allocation for partition_shapes failed");
        return;
    }
    cudaMemcpy(d_rp, csrRow, sizeof(int) * ((size_t)M + 1), cudaMemcpyHostToDevice);
    if (nz) {
        cudaMemcpy(d_col, csrCol, sizeof(int) * nz, cudaMemcpyHostToDevice);
        cudaMemcpy(d_val, csrVal, sizeof(float) * nz, cudaMemcpyHostToDevice);
    }
    tc::PartitionOut po;
    double t0 = now_ms();
    tc_status st = tc::gpu_partition(M, N, nnz, d_rp, d_col, d_val, prm, false, true, 0, po);
    double t1 = now_ms();
    cudaFree(d_rp); cudaFree(d_col); cudaFree(d_val);
    if (st != TC_OK) {
        printf("CUDA Runtime Error: %s\n", tc_last_error());
        if (po.d_rowptr) cudaFree(po.d_rowptr);
        if (po.d_cols) cudaFree(po.d_cols);
        return;
    }
    // the reference's FLT_MAX marks on claimed entries (TaiChi.cu:866)
    for (size_t j = 0; j < po.claimed.size() && j < nz; ++j)
        if (po.claimed[j]) csrVal[j] = FLT_MAX;
    printf("dia_shapes=%d, num_negs=%d, dense_nnz=%d, sparse_nnz=%d\n", po.dia_shapes, po.num_negs,
           po.dense_nnz, po.sparse_nnz);
    t->dia_shapes = po.dia_shapes; t->num_negs = po.num_negs; t->dense_nnz = po.dense_nnz;
    t->zero_elements = po.zero_elements; t->sparse_nnz = po.sparse_nnz;
    t->row_start = po.row_start; t->row_stop = po.row_stop;
    auto dup = [](const std::vector<int> &v) -> int * {
        if (v.empty()) return nullptr;
        int *p = (int *)malloc(v.size() * sizeof(int));
        memcpy(p, v.data(), v.size() * sizeof(int));
        return p;
    };
    if (po.dia_shapes > 0) {
        t->xStart = dup(po.xStart); t->yStart = dup(po.yStart); t->xStop = dup(po.xStop);
        t->nDiasPtr = dup(po.nDiasPtr); t->neg_offsets = dup(po.offsets);
    }
    if (po.aliases_input) {
        t->csrRow = csrRow;
        t->csrCol = csrCol;
    } else if (po.nnz_csr > 0) {
        t->csrRow = (int *)malloc(sizeof(int) * ((size_t)M + 1));
        t->csrCol = (int *)malloc(sizeof(int) * (size_t)po.nnz_csr);
        cudaMemcpy(t->csrRow, po.d_rowptr, sizeof(int) * ((size_t)M + 1), cudaMemcpyDeviceToHost);
        cudaMemcpy(t->csrCol, po.d_cols, sizeof(int) * (size_t)po.nnz_csr, cudaMemcpyDeviceToHost);
    }
    if (po.d_rowptr) cudaFree(po.d_rowptr);
    if (po.d_cols) cudaFree(po.d_cols);
    printf("getSdf:%.4f partition_dense:%.4f partition_sparse:%.4f ms\n", po.ms, t1 - t0 - po.ms, 0.0);
}

// TaiChi.cu:1331-1456: uploads the format, runs warm-up and timed launches,
// prints the mean transfer and multiply times, and returns y.
void taichi_SpMV(int M, int N, TaiChi_new *t, float *xHost, float *yHost)
{
    if (!t) return;
    tc_format f{};
    f.dia_shapes = t->dia_shapes; f.num_negs = t->num_negs; f.dense_nnz = t->dense_nnz;
    f.zero_elements = t->zero_elements; f.sparse_nnz = t->sparse_nnz;
    f.row_start = t->row_start; f.row_stop = t->row_stop;
    f.xStart = t->xStart; f.yStart = t->yStart; f.xStop = t->xStop;
    f.nDiasPtr = t->nDiasPtr; f.neg_offsets = t->neg_offsets;
    f.csrRow = t->csrRow; f.csrCol = t->csrCol;
    const int nrun = env_int("TAICHI_B200_NUM_RUN", NUM_RUN);
    const int ntransfer = std::max(1, env_int("TAICHI_B200_NUM_TRANSFER", NUM_TRANSFER));
    tc_plan *p = nullptr;
    double tt = 0.0;
    for (int i = 0; i < ntransfer; ++i) {   // format upload, timed like the reference
        if (p) tc_plan_destroy(p);
        p = nullptr;
        double a = now_ms();
        tc_status st = tc_plan_from_format(M, N, &f, nullptr, 0, &p);
        tt += now_ms() - a;
        if (st != TC_OK) {
            printf("CUDA Runtime Error: %s\n", tc_last_error());
            return;
        }
    }
    float *dx = nullptr, *dy = nullptr;
    if (cudaMalloc(&dx, sizeof(float) * ((size_t)N + 4)) != cudaSuccess ||
        cudaMalloc(&dy, sizeof(float) * ((size_t)M + 4)) != cudaSuccess) {
        printf("CUDA Runtime Error: %s\n", "allocation of x / y failed");
        tc_plan_destroy(p);
        return;
    }
    cudaMemcpy(dx, xHost, sizeof(float) * (size_t)N, cudaMemcpyHostToDevice);
    // every multiply's status is checked; the first failure is printed the way
    // the reference prints a CUDA error (TaiChi.cu:42-55) and y is left as is
    tc_status st = TC_OK;
    for (int i = 0; i < 10 && st == TC_OK; ++i) st = tc_spmv(p, dx, dy, 0);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double total = 0.0;
    for (int i = 0; i < nrun && st == TC_OK; ++i) {
        cudaEventRecord(e0, 0);
        st = tc_spmv(p, dx, dy, 0);
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        total += ms;
    }
    if (nrun == 0 && st == TC_OK) st = tc_spmv(p, dx, dy, 0);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st == TC_OK) st = tc_plan_check(p);     // a device-side give-up leaves y incomplete
    if (st == TC_OK && cudaDeviceSynchronize() != cudaSuccess)
        st = tc::fail(TC_ERR_CUDA, "multiply: %s", cudaGetErrorString(cudaGetLastError()));
    if (st != TC_OK) {
        printf("CUDA Runtime Error: %s\n", tc_last_error());
        cudaFree(dx);
        cudaFree(dy);
        tc_plan_destroy(p);
        return;
    }
    printf("transfer_time:%.4f spmv_time=%.4f\n", tt / ntransfer, nrun ? total / nrun : 0.0);
    cudaMemcpy(yHost, dy, sizeof(float) * (size_t)M, cudaMemcpyDeviceToHost);
    cudaFree(dx);
    cudaFree(dy);
    tc_plan_destroy(p);
    if (env_int("TAICHI_B200_DEVICE_RESET", 0)) cudaDeviceReset();
}
