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
constexpr int kErrBulkArg = 2;  // a bulk copy failed its alignment / bounds check

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

// 1-D bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned)
// from this CTA's shared memory to global, tracked by the issuing thread's
// bulk group.  The writers of the source must have executed
// fence_proxy_async_smem() and a CTA barrier before the issue.
__device__ __forceinline__ void bulk_copy_s2g(void* dst, const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_addr(src)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Until the sources of this thread's committed bulk stores have been read
// (the shared memory may be reused or released afterwards).
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }

// Hint: bring `bytes` (multiple of 16, 16-byte aligned) of global memory into
// L2 ahead of a later bulk copy.
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ uint32_t dynamic_smem_bytes() {
    uint32_t v;
    asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(v));
    return v;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Checks a bulk copy against the rules it must meet: both addresses 16-byte
// aligned, the size a non-zero multiple of 16, the shared-memory side inside
// the CTA's dynamic shared memory (`smem_base` is its start).  On failure it
// records kErrBulkArg in *err and returns false, and the caller skips the copy.
__device__ __forceinline__ bool bulk_args_ok(const void* gptr, const void* sptr, uint32_t bytes,
                                             const void* smem_base, int* err) {
    const uint32_t off = smem_addr(sptr) - smem_addr(smem_base);
    const bool ok = ((reinterpret_cast<uintptr_t>(gptr) | off | bytes) & 15u) == 0 && bytes != 0 &&
                    off + bytes <= dynamic_smem_bytes() && off + bytes >= off;
    if (!ok && err) atomicExch(err, kErrBulkArg);
    return ok;
}

// Global -> shared bulk copy completing on `bar`, after the checks above; a
// copy that fails them is replaced by a plain arrive, so the waiters still
// finish (on stale data, with the error recorded).
__device__ __forceinline__ void bulk_load_checked(void* dst, const void* src, uint32_t bytes, uint64_t* bar,
                                                  const void* smem_base, int* err) {
    if (bulk_args_ok(src, dst, bytes, smem_base, err)) {
        mbar_arrive_expect_tx(bar, bytes);
        bulk_copy_g2s(dst, src, bytes, bar);
    } else {
        mbar_arrive(bar);
    }
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
// the budget (SM clock cycles) ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err,
                                          long long budget = kWaitBudgetCycles) {
    const long long start = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - start > budget) {
            if (err) atomicExch(err, kErrWaitTimeout);
            return false;
        }
    }
    return true;
}

}  // namespace ld
