// tc_scan.cuh -- device-wide exclusive prefix sum of int32 (used by the
// partitioner's compactions and the device format build).  Two-level
// reduce-then-scan with 4096 elements per 256-thread block; recursion on the
// block totals.  The kernels have internal linkage: each file that includes
// this header gets its own copies.
#pragma once

#include <cuda_runtime.h>

#include "tc_internal.h"

namespace tc {
namespace scan_detail {
namespace {

constexpr int kThreads = 256;
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;   // 4096

__device__ __forceinline__ int block_exclusive(int v, int *sh, int *total)
{
    // warp-level inclusive scan, then warp totals
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int t = lane < kThreads / 32 ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < kThreads / 32) sh[lane] = t;   // inclusive warp totals
    }
    __syncthreads();
    const int before = warp ? sh[warp - 1] : 0;
    *total = sh[kThreads / 32 - 1];
    __syncthreads();
    return before + x - v;
}

// out[i] = sum(in[0..i)), tile-local; tile totals into sums[blockIdx.x].
__global__ void scan_tiles(const int *__restrict__ in, int *__restrict__ out, int n,
                           int *__restrict__ sums)
{
    __shared__ int sh[kThreads / 32];
    const int base = blockIdx.x * kTile + threadIdx.x * kItems;
    int v[kItems];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        v[k] = base + k < n ? in[base + k] : 0;
        s += v[k];
    }
    int total;
    int run = block_exclusive(s, sh, &total);
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (sums && threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void add_offsets(int *__restrict__ out, int n, const int *__restrict__ offs)
{
    const int base = blockIdx.x * kTile;
    const int add = offs[blockIdx.x];
    for (int i = threadIdx.x; i < kTile && base + i < n; i += kThreads) out[base + i] += add;
}

}  // namespace
}  // namespace scan_detail

// Exclusive scan of n ints; writes n+1 values (out[n] = total).  `tmp` must
// hold scan_tmp_ints(n) ints.  in and out may alias.
static inline size_t scan_tmp_ints(long n)
{
    size_t t = 0;
    long m = n + 1;
    while (m > scan_detail::kTile) {
        m = (m + scan_detail::kTile - 1) / scan_detail::kTile;
        t += 2 * (size_t)m + 2;
    }
    return t + 2;
}

static inline tc_status exclusive_scan(const int *in, int *out, long n, int *tmp, cudaStream_t s)
{
    using namespace scan_detail;
    // treat the input as n+1 values with a trailing 0 so out[n] is the total
    // (the caller guarantees in[n] readable and zero, or in == out with
    // out[n] zero).
    const long m = n + 1;
    const int blocks = (int)((m + kTile - 1) / kTile);
    if (blocks == 1) {
        scan_tiles<<<1, kThreads, 0, s>>>(in, out, (int)m, nullptr);
        TC_CUDA(cudaGetLastError());
        return TC_OK;
    }
    int *sums = tmp;
    int *rest = tmp + blocks + 1;
    scan_tiles<<<blocks, kThreads, 0, s>>>(in, out, (int)m, sums);
    TC_CUDA(cudaGetLastError());
    TC_CUDA(cudaMemsetAsync(sums + blocks, 0, sizeof(int), s));
    TC_CHECK(exclusive_scan(sums, sums, blocks, rest, s));
    add_offsets<<<blocks, kThreads, 0, s>>>(out, (int)m, sums);
    TC_CUDA(cudaGetLastError());
    return TC_OK;
}

}  // namespace tc
