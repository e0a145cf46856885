// adapter_harness.cpp — TEST INFRASTRUCTURE: drives the drop-in adapter
// (lensdiff_b200/adapter/LensDiffCudaB200.cpp) through the reference's own
// request / parameter types, the way the plugin calls it at
// source/src/LensDiff.cpp:3833.  Built by oracle/Makefile into
// oracle/_ref/libldadapter.so together with the adapter and the reference's
// spectrum / colour sources (the adapter calls the plugin's
// BuildLensDiffSpectrumConfig); linked with liblensdiff_b200.so.
#include "LensDiffTypes.h"
#include "lensdiff_b200.h"
#include "ref_params.h"

#include <cstring>
#include <string>

bool RunLensDiffCuda(const LensDiffRenderRequest& request, const LensDiffParams& params,
                     LensDiffPsfBankCache& cache, std::string* error);

extern "C" int ldadapter_render(const ld_params* p, void* src_dev, int sx1, int sy1, int sw, int sh,
                                long long src_row_bytes, void* dst_dev, int dx1, int dy1, int dw, int dh,
                                long long dst_row_bytes, int rx1, int ry1, int rx2, int ry2, void* stream,
                                int host_enabled, char* error, int error_cap) {
    LensDiffRenderRequest req {};
    req.renderWindow = {rx1, ry1, rx2, ry2};
    req.frameBounds = {sx1, sy1, sx1 + sw, sy1 + sh};
    req.src.data = src_dev;
    req.src.rowBytes = static_cast<std::ptrdiff_t>(src_row_bytes);
    req.src.bounds = {sx1, sy1, sx1 + sw, sy1 + sh};
    req.dst.data = dst_dev;
    req.dst.rowBytes = static_cast<std::ptrdiff_t>(dst_row_bytes);
    req.dst.bounds = {dx1, dy1, dx1 + dw, dy1 + dh};
    req.frameShortSidePx = p->frame_short_side_px;
    req.hostEnabledCudaRender = host_enabled != 0;
    req.cudaStream = stream;
    LensDiffPsfBankCache cache {};
    std::string err;
    const bool ok = RunLensDiffCuda(req, toReference(*p), cache, &err);
    if (error && error_cap > 0) {
        std::strncpy(error, err.c_str(), static_cast<std::size_t>(error_cap - 1));
        error[error_cap - 1] = '\0';
    }
    return ok ? 1 : 0;
}
