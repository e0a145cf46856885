// ref_cuda_harness.cpp — TEST INFRASTRUCTURE: drives the reference's own CUDA
// chain, RunLensDiffCuda (source/src/cuda/LensDiffCuda.cu:4642-7587, compiled
// unchanged for sm_100a with the VkFFT stub, so its transforms run on cuFFT),
// through the reference's request and parameter types, as the plugin calls it
// at source/src/LensDiff.cpp:3833.  Built by oracle/Makefile into
// oracle/_ref/libldrefcuda.so.  It is the comparator the library's frame
// rates are set against on the same GPU; nothing of the library runs here.
//
// The plugin keeps one LensDiffPsfBankCache per effect instance across frames
// (LensDiff.cpp:3833); `instance` selects one of a few such caches kept here,
// so repeated calls see the reference's own caching.
#include "LensDiffCuda.h"
#include "LensDiffTypes.h"
#include "lensdiff_b200.h"
#include "ref_params.h"

#include <cstring>
#include <string>

namespace {
LensDiffPsfBankCache g_caches[4];
}

extern "C" int ldrefcuda_render(const ld_params* p, int instance, void* src_dev, int width, int height,
                                long long row_bytes, void* dst_dev, void* stream, char* error, int error_cap) {
    if (instance < 0 || instance >= 4) return 0;
    LensDiffRenderRequest req {};
    req.renderWindow = {0, 0, width, height};
    req.frameBounds = {0, 0, width, height};
    req.src.data = src_dev;
    req.src.rowBytes = static_cast<std::ptrdiff_t>(row_bytes);
    req.src.bounds = {0, 0, width, height};
    req.dst.data = dst_dev;
    req.dst.rowBytes = static_cast<std::ptrdiff_t>(row_bytes);
    req.dst.bounds = {0, 0, width, height};
    req.frameShortSidePx = p->frame_short_side_px;
    req.hostEnabledCudaRender = true;
    req.cudaStream = stream;
    std::string err;
    const bool ok = RunLensDiffCuda(req, toReference(*p), g_caches[instance], &err);
    if (error && error_cap > 0) {
        std::strncpy(error, err.c_str(), static_cast<std::size_t>(error_cap - 1));
        error[error_cap - 1] = '\0';
    }
    return ok ? 1 : 0;
}
