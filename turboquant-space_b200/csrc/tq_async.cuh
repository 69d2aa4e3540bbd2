// tq_async.cuh -- mbarrier and bulk-copy helpers shared by the sm_100a kernels
// (tq_kernels.cu, tq_tc.cu).  Device-only, header-only.
//
// Every wait on an mbarrier is bounded: after kWaitCycles the waiting thread
// records an error code in a device status word and gives up, so that a copy
// or an arrive that never comes ends in an error status instead of a hung GPU.
#pragma once

#include <cstdint>

namespace tq {

constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 2 GHz

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// Makes mbarrier initialisation visible to the async proxy (bulk copies).
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: true when the phase completed; false after the budget ran out
// (error recorded) or when another thread already recorded an error.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int *err, int code) {
    const long long t0 = clock64();
    for (uint32_t it = 1;; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 1023u) == 0) {
            if (*reinterpret_cast<volatile int *>(err) != 0) return false;
            if (clock64() - t0 > kWaitCycles) {
                atomicCAS(err, 0, code);
                return false;
            }
        }
    }
}

// Bounded wait that ignores the status word: used to drain this thread's own
// copies in flight before it exits after an error.
__device__ __forceinline__ bool mbar_drain(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    for (uint32_t it = 1;; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 1023u) == 0 && clock64() - t0 > kWaitCycles) return false;
    }
}

// Orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy operations (a bulk copy that overwrites the buffer).
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Untiled bulk copy global -> this CTA's shared memory, completing `bytes` of
// transaction count on `bar`.  dst, src and bytes must be multiples of 16.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes,
                                          uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(bar)
        : "memory");
}

}  // namespace tq
