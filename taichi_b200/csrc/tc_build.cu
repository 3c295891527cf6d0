// tc_build.cu -- format build on the device: Matrix Market entries (parsed on
// the host) -> CSR in device memory, with readMtx's row order.
//
// readMtx (TaiChi.cu:170-270) places every entry with a counting sort in file
// order: entry i goes to the end of row i_row, and in a symmetric (or
// hermitian) file an off-diagonal entry is followed, at the same step, by its
// mirror at the end of row i_col.  So within a row the entries are ordered by
// their file index, a direct entry and a mirror alike.  Here every file entry
// i contributes two sort records, (row, 2i) and (column, 2i + 1) for a mirror
// or (M, 2i + 1) -- a key past every row -- when it has none.  A stable least
// significant digit radix sort of the records by key (8-bit digits; a block
// ranks its records in index order with warp match masks) leaves each row's
// records in file order, mirrors where readMtx puts them; the first nnz
// records are the matrix.  A gather then writes the columns and values, and a
// row histogram with a prefix sum the row pointers.  The text parse stays on
// the host (tc_mtx.cpp); this file replaces the host counting sort.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>

#include "tc_internal.h"
#include "tc_scan.cuh"

namespace tc {
namespace {

constexpr int kSortThreads = 256;
constexpr int kSortRounds = 8;                         // rounds of 256 records per block
constexpr int kSortTile = kSortThreads * kSortRounds;  // records per block
constexpr int kRadix = 256;

long cdivl(long a, long b) { return (a + b - 1) / b; }

// Sort records from the file entries: record 2i = (row of entry i, 2i),
// record 2i + 1 = (column of entry i, 2i + 1) if it is an off-diagonal entry
// of a symmetric file, else (M, 2i + 1).
__global__ void make_records(const MtxEntry *__restrict__ e, long n, int M, int symmetric,
                             unsigned *__restrict__ key, unsigned *__restrict__ idx)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const MtxEntry en = e[i];
    key[2 * i] = (unsigned)(en.i - 1);
    idx[2 * i] = (unsigned)(2 * i);
    key[2 * i + 1] = symmetric && en.i != en.j ? (unsigned)(en.j - 1) : (unsigned)M;
    idx[2 * i + 1] = (unsigned)(2 * i + 1);
}

// Per block, the count of each digit of its tile: hist[d * nblocks + block]
// (digit-major, so an exclusive scan gives each block's first slot per digit).
__global__ void __launch_bounds__(kSortThreads) radix_hist(const unsigned *__restrict__ key, long n, int shift,
                                                           unsigned *__restrict__ hist)
{
    __shared__ unsigned cnt[kRadix];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    const long base = (long)blockIdx.x * kSortTile;
    for (int r = 0; r < kSortRounds; ++r) {
        const long i = base + r * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&cnt[(key[i] >> shift) & (kRadix - 1)], 1u);
    }
    __syncthreads();
    hist[(long)threadIdx.x * gridDim.x + blockIdx.x] = cnt[threadIdx.x];
}

// Stable scatter of one digit pass: each block walks its tile in index order
// (steps of 256 records); a record's slot is its block's first slot for its
// digit, plus the records of that digit in earlier steps, earlier warps of
// this step, and earlier lanes of its warp.
__global__ void __launch_bounds__(kSortThreads) radix_scatter(const unsigned *__restrict__ key_in,
                                                              const unsigned *__restrict__ idx_in, long n,
                                                              int shift, const unsigned *__restrict__ offs,
                                                              unsigned *__restrict__ key_out,
                                                              unsigned *__restrict__ idx_out)
{
    constexpr int kWarps = kSortThreads / 32;
    __shared__ unsigned slot[kRadix];                // next slot of each digit
    __shared__ unsigned wcnt[kWarps][kRadix];        // this step's count per warp and digit
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    slot[threadIdx.x] = offs[(long)threadIdx.x * gridDim.x + blockIdx.x];
    const long base = (long)blockIdx.x * kSortTile;
    const unsigned lt = (1u << lane) - 1u;
    for (int r = 0; r < kSortRounds; ++r) {
        for (int w = 0; w < kWarps; ++w) wcnt[w][threadIdx.x] = 0;
        __syncthreads();
        const long i = base + r * kSortThreads + threadIdx.x;
        const bool ok = i < n;
        const unsigned k = ok ? key_in[i] : 0u, v = ok ? idx_in[i] : 0u;
        const unsigned d = ok ? (k >> shift) & (kRadix - 1) : kRadix;     // kRadix: no record
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const unsigned rank = __popc(peers & lt);
        if (ok && rank == 0) wcnt[warp][d] = __popc(peers);
        __syncthreads();
        if (ok) {
            unsigned before = 0;
            for (int w = 0; w < warp; ++w) before += wcnt[w][d];
            const unsigned at = slot[d] + before + rank;
            key_out[at] = k;
            idx_out[at] = v;
        }
        __syncthreads();
        unsigned tot = 0;                             // thread t advances digit t
        for (int w = 0; w < kWarps; ++w) tot += wcnt[w][threadIdx.x];
        slot[threadIdx.x] += tot;
    }
}

__global__ void row_counts(const unsigned *__restrict__ key, long nnz, int *__restrict__ cnt)
{
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < nnz) atomicAdd(cnt + key[p], 1);
}

__global__ void gather_entries(const unsigned *__restrict__ idx, long nnz, const MtxEntry *__restrict__ e,
                               int *__restrict__ col, float *__restrict__ val)
{
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nnz) return;
    const unsigned v = idx[p];
    const MtxEntry en = e[v >> 1];
    col[p] = (v & 1u) ? en.i - 1 : en.j - 1;    // a mirror's column is the entry's row
    val[p] = en.v;
}

struct Buf {
    void *p = nullptr;
    ~Buf() { if (p) cudaFree(p); }
    tc_status alloc(size_t bytes)
    {
        const cudaError_t e = cudaMalloc(&p, std::max<size_t>(bytes, 16));
        if (e != cudaSuccess) {
            p = nullptr;
            return fail(TC_ERR_ALLOC, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
        }
        return TC_OK;
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
    void *release() { void *q = p; p = nullptr; return q; }
};

double ms_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

// Device CSR from file-order entries (1-based, already checked against M x N).
tc_status coo_to_csr_device(int M, int N, bool symmetric, const MtxEntry *h_entries, long n, cudaStream_t s,
                            int **d_rowptr, int **d_col, float **d_val, int64_t *nnz_out)
{
    (void)N;
    Buf ent, keyA, keyB, idxA, idxB, hist, tmp, rp, cl, vl;
    const long nrec = 2 * n;
    if (nrec > 0x7fffffffL) return fail(TC_ERR_UNSUPPORTED, "more than 2^30 file entries");
    TC_CHECK(ent.alloc(sizeof(MtxEntry) * (size_t)n));
    TC_CHECK(keyA.alloc(sizeof(unsigned) * (size_t)nrec));
    TC_CHECK(keyB.alloc(sizeof(unsigned) * (size_t)nrec));
    TC_CHECK(idxA.alloc(sizeof(unsigned) * (size_t)nrec));
    TC_CHECK(idxB.alloc(sizeof(unsigned) * (size_t)nrec));
    const long blocks = std::max(1L, cdivl(nrec, kSortTile));
    const long nh = blocks * kRadix;
    TC_CHECK(hist.alloc(sizeof(unsigned) * (size_t)(nh + 1)));
    TC_CHECK(tmp.alloc(sizeof(int) * scan_tmp_ints(std::max<long>(nh, (long)M + 1))));
    TC_CHECK(rp.alloc(sizeof(int) * ((size_t)M + 2)));
    if (n) TC_CUDA(cudaMemcpyAsync(ent.p, h_entries, sizeof(MtxEntry) * (size_t)n, cudaMemcpyHostToDevice, s));
    if (n) {
        make_records<<<(unsigned)cdivl(n, 256), 256, 0, s>>>(ent.as<MtxEntry>(), n, M, symmetric ? 1 : 0,
                                                            keyA.as<unsigned>(), idxA.as<unsigned>());
        TC_CUDA(cudaGetLastError());
    }
    // keys run up to M (the "no mirror" key), so the passes cover M's bits
    int bits = 1;
    while (bits < 32 && ((unsigned)M >> bits) != 0) ++bits;
    unsigned *ki = keyA.as<unsigned>(), *ko = keyB.as<unsigned>();
    unsigned *ii = idxA.as<unsigned>(), *io = idxB.as<unsigned>();
    for (int shift = 0; shift < bits && nrec > 0; shift += 8) {
        radix_hist<<<(unsigned)blocks, kSortThreads, 0, s>>>(ki, nrec, shift, hist.as<unsigned>());
        TC_CUDA(cudaGetLastError());
        TC_CUDA(cudaMemsetAsync(hist.as<unsigned>() + nh, 0, sizeof(unsigned), s));   // the scan's trailing 0
        TC_CHECK(exclusive_scan(hist.as<int>(), hist.as<int>(), nh, tmp.as<int>(), s));
        radix_scatter<<<(unsigned)blocks, kSortThreads, 0, s>>>(ki, ii, nrec, shift, hist.as<unsigned>(), ko, io);
        TC_CUDA(cudaGetLastError());
        std::swap(ki, ko);
        std::swap(ii, io);
    }
    // nnz = records with a key below M
    int64_t nnz = n;
    if (symmetric) {
        nnz = 0;
        for (long i = 0; i < n; ++i) nnz += h_entries[i].i != h_entries[i].j ? 2 : 1;
    }
    if (nnz > 0x7fffffffL) return fail(TC_ERR_UNSUPPORTED, "more than 2^31 entries");
    TC_CHECK(cl.alloc(sizeof(int) * (size_t)std::max<int64_t>(nnz, 1)));
    TC_CHECK(vl.alloc(sizeof(float) * (size_t)std::max<int64_t>(nnz, 1)));
    TC_CUDA(cudaMemsetAsync(rp.p, 0, sizeof(int) * ((size_t)M + 2), s));
    if (nnz) {
        row_counts<<<(unsigned)cdivl(nnz, 256), 256, 0, s>>>(ki, nnz, rp.as<int>());
        gather_entries<<<(unsigned)cdivl(nnz, 256), 256, 0, s>>>(ii, nnz, ent.as<MtxEntry>(), cl.as<int>(),
                                                                vl.as<float>());
        TC_CUDA(cudaGetLastError());
    }
    TC_CHECK(exclusive_scan(rp.as<int>(), rp.as<int>(), M, tmp.as<int>(), s));
    TC_CUDA(cudaStreamSynchronize(s));
    *d_rowptr = static_cast<int *>(rp.release());
    *d_col = static_cast<int *>(cl.release());
    *d_val = static_cast<float *>(vl.release());
    *nnz_out = nnz;
    return TC_OK;
}

}  // namespace tc

extern "C" {

tc_status tc_read_mtx_device(const char *path, int *M, int *N, int64_t *nnz, int **d_rowptr, int **d_col,
                             float **d_val, int *ref_code, double *parse_ms, double *build_ms, void *stream)
{
    int dummy;
    if (!ref_code) ref_code = &dummy;
    *ref_code = 0;
    if (!path || !M || !N || !nnz || !d_rowptr || !d_col || !d_val)
        return tc::fail(TC_ERR_INVALID, "tc_read_mtx_device: null argument");
    const auto t0 = std::chrono::steady_clock::now();
    tc::MtxCoo coo;
    TC_CHECK(tc::mtx_parse(path, coo, ref_code));
    if (parse_ms) *parse_ms = tc::ms_since(t0);
    const auto t1 = std::chrono::steady_clock::now();
    TC_CHECK(tc::coo_to_csr_device(coo.M, coo.N, coo.symmetric, coo.entries.data(), (long)coo.entries.size(),
                                   (cudaStream_t)stream, d_rowptr, d_col, d_val, nnz));
    if (build_ms) *build_ms = tc::ms_since(t1);
    *M = coo.M;
    *N = coo.N;
    return TC_OK;
}

void tc_device_free(void *p)
{
    if (p) cudaFree(p);
}

}  // extern "C"
