// vkfft_stub.cpp — TEST INFRASTRUCTURE: stands in for the reference's VkFFT
// translation unit (source/src/cuda/LensDiffCudaVkFFT.cu), whose third-party
// VkFFT headers (a git submodule at an unrecorded commit) are absent.  Every
// plan request fails, so the reference's own CUDA chain takes its cuFFT
// fallback (LensDiffCuda.cu:2569-2576, :2611-2628) and can be timed here.
#include "LensDiffCudaVkFFT.h"

LensDiffCudaVkFFTPlanLease::LensDiffCudaVkFFTPlanLease(LensDiffCudaVkFFTPlanLease&& other) noexcept
    : repository(other.repository), entry(other.entry), releaseStream(other.releaseStream),
      persistent(other.persistent) {
    other.repository = nullptr;
    other.entry = nullptr;
}

LensDiffCudaVkFFTPlanLease& LensDiffCudaVkFFTPlanLease::operator=(LensDiffCudaVkFFTPlanLease&& other) noexcept {
    repository = other.repository;
    entry = other.entry;
    releaseStream = other.releaseStream;
    persistent = other.persistent;
    other.repository = nullptr;
    other.entry = nullptr;
    return *this;
}

LensDiffCudaVkFFTPlanLease::~LensDiffCudaVkFFTPlanLease() = default;

void LensDiffCudaVkFFTPlanLease::release() {
    repository = nullptr;
    entry = nullptr;
}

std::size_t LensDiffCudaVkFFTPlanLease::workBytes() const { return 0; }

bool lensDiffCudaVkFFTAcquirePlan(bool, int, int, int, int, cudaStream_t, double* outInitMs, bool* outCacheHit,
                                  LensDiffCudaVkFFTPlanLease*, std::string* error) {
    if (outInitMs) *outInitMs = 0.0;
    if (outCacheHit) *outCacheHit = false;
    if (error) *error = "vkfft-not-built";
    return false;
}

bool lensDiffCudaVkFFTExecC2C(LensDiffCudaVkFFTPlanLease*, void*, bool, std::string* error) {
    if (error) *error = "vkfft-not-built";
    return false;
}
