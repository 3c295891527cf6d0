/*
 * Build shim for compiling the reference's TaiChi.cu without the CUSP
 * library.  TaiChi.cu:1275 and morohutils.cu:219 only ask CUSP for the number
 * of thread blocks of a kernel that can be resident on the whole device; the
 * CUDA runtime answers that directly.  Test infrastructure only.
 */
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

namespace cusp { namespace system { namespace cuda { namespace detail {
template <typename Kernel>
inline size_t max_active_blocks(Kernel kernel, size_t block_threads, size_t dyn_smem)
{
    int per_sm = 0, dev = 0, sms = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, (int)block_threads, dyn_smem);
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (size_t)per_sm * (size_t)sms;
}
}}}}
