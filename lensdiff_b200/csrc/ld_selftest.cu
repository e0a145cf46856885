// ld_selftest.cu — device-side failure detection, exercised without a fault.
//
// The library's kernels wait on shared-memory mbarriers for bulk copies, and
// every such wait is bounded (mbar_wait, ld_async.cuh): a copy that never
// completes makes the wait give up, record an error in the context's device
// error word and return, so the context stays usable.  Likewise a bulk copy
// whose arguments break the copy engine's rules is never issued
// (bulk_load_checked).  This kernel drives those two paths on purpose, with
// nothing that could fault the GPU: the timeout case waits on a barrier that
// no copy and no thread will ever complete, with a caller-given budget of SM
// clock cycles; the argument case asks for a copy of 20 bytes (not a multiple
// of 16), which the check refuses before anything is issued.  A third case
// runs one valid copy and must record nothing.  No bulk copy is in flight
// when the kernel returns in any case.
#include "../../include/lensdiff_b200.h"
#include "ld_async.cuh"
#include "ld_internal.h"

namespace ld {
namespace {

// one CTA of 64 threads; dynamic shared memory: 64 float4 + the barrier
__global__ void __launch_bounds__(64) wait_selftest_kernel(int mode, long long budget, const float4* src, float4* dst,
                                                           int* err) {
    extern __shared__ __align__(128) unsigned char smraw[];
    float4* buf = reinterpret_cast<float4*>(smraw);
    uint64_t* bar = reinterpret_cast<uint64_t*>(buf + 64);
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (mode == LD_SELFTEST_BAD_COPY_ARGS) {
            bulk_load_checked(buf, src, 20u, bar, smraw, err);  // refused: 20 is not a multiple of 16
        } else if (mode == LD_SELFTEST_VALID_COPY) {
            bulk_load_checked(buf, src, 64u * sizeof(float4), bar, smraw, err);
        }
        // LD_SELFTEST_WAIT_TIMEOUT: nothing arrives on the barrier
    }
    const bool ok = mbar_wait(bar, 0, err, budget);
    if (__syncthreads_or(!ok)) return;
    if (mode == LD_SELFTEST_VALID_COPY) dst[threadIdx.x] = buf[threadIdx.x];
}

}  // namespace

int launch_wait_selftest(int mode, long long budget, float4* scratch, int* err, cudaStream_t s) {
    if (mode != LD_SELFTEST_WAIT_TIMEOUT && mode != LD_SELFTEST_BAD_COPY_ARGS && mode != LD_SELFTEST_VALID_COPY)
        return LD_ERR_ARG;
    // at least ~1 us, at most the library's own wait budget
    if (budget < 1000 || budget > kWaitBudgetCycles) return LD_ERR_ARG;
    const size_t smem = 64 * sizeof(float4) + sizeof(uint64_t);
    wait_selftest_kernel<<<1, 64, smem, s>>>(mode, budget, scratch, scratch + 64, err);
    return cudaGetLastError() == cudaSuccess ? LD_OK : LD_ERR_CUDA;
}

}  // namespace ld
