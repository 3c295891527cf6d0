// tc_tma.cuh -- bulk asynchronous copies (TMA, cp.async.bulk) into shared
// memory with completion on an mbarrier, and the bounded waits on them.
// Shared by the multiply kernels that stage their operands.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace tc {

__device__ __forceinline__ unsigned smem_u32(const void *p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *m, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *m, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(m)),
                 "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, uint64_t *m)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(m)) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t *m, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}" : "=r"(ok) : "r"(smem_u32(m)), "r"(parity) : "memory");
    return ok != 0;
}
// Nanoseconds of the GPU's global timer.
__device__ __forceinline__ uint64_t globaltimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait: gives up once kStageWaitNs of global-timer time have passed
// since the first failed poll (the copies complete in microseconds; a
// give-up is reported through the plan's error word).  The deadline is time,
// not a poll count, because each try_wait may suspend the thread for a
// hardware-chosen interval.
constexpr uint64_t kStageWaitNs = 1000000000ull;   // 1 s

__device__ __forceinline__ bool mbar_wait(uint64_t *m, unsigned parity)
{
    if (mbar_test(m, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    for (;;) {
        for (int i = 0; i < 32; ++i)
            if (mbar_test(m, parity)) return true;
        if (globaltimer_ns() - t0 > kStageWaitNs) return false;
    }
}
__device__ __forceinline__ void fence_async_shared()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 16-byte aligned byte window [a, b) that covers elements [e0, e1) of an
// int array (the plan arrays are padded, so the window stays inside them).
struct Window {
    long a, b;
    int shift;   // index of element e0 inside the window
};
__device__ __forceinline__ Window window_of(long e0, long e1)
{
    Window w;
    w.a = (e0 * 4) & ~15L;
    w.b = (e1 * 4 + 15) & ~15L;
    w.shift = (int)((e0 * 4 - w.a) >> 2);
    return w;
}

}  // namespace tc
