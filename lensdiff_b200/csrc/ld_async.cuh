// ld_async.cuh — bulk asynchronous global->shared copies (the TMA bulk-copy
// engine, cp.async.bulk) completed through shared-memory mbarriers, with
// bounded waits.
//
// Every wait gives up after a clock budget (about a second), records the
// failure in a device error word and reports it to the caller, so a copy that
// never lands cannot hang the GPU; the host reads the error word with
// ld_check_device_errors.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ld {

constexpr long long kWaitBudgetCycles = 2000000000LL;  // ~1 s at 1.9 GHz
constexpr int kErrWaitTimeout = 1;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes the barrier initialisation visible to the async (bulk copy) proxy.
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy accesses (a bulk copy about to overwrite a buffer).
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// 1-D bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned)
// from global to this CTA's shared memory; completes on `bar`.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of `bar`.  Returns false (and sets *err) if
// the budget ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
    const long long start = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - start > kWaitBudgetCycles) {
            if (err) atomicExch(err, kErrWaitTimeout);
            return false;
        }
    }
    return true;
}

}  // namespace ld
