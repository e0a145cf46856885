// ld_noalloc.cu — raw-PSF entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc: an OpenFX host that owns the GPU's
// memory and budgets it for the whole node graph, a real-time playback thread
// that must not take cudaMalloc's implicit device synchronisation, or an
// embedding that runs under a fixed, pre-reserved memory budget.  For them
// ld_raw_psf_noalloc computes the same normalised, fft-shifted raw PSF as
// ld_raw_psf without a context and without any allocation: its scratch (the
// twiddle table, the pupil pre-pass, the row-pass output and the energy sum)
// lives in the file-scope device array below, of a fixed size.
//
// Limits and sharing:
//   * the array holds kNoAllocScratchBytes (12 MiB) on every GPU that loads the
//     library, for the life of the process;
//   * sizes beyond it (pupil > 512 or PSF grid > 1024, i.e. a maximum kernel
//     radius above 256 px) are rejected with LD_ERR_ARG and a stage string;
//   * every call on a device uses the same array, which keeps the previous
//     call's contents; the energy sum is cleared at the start of each call.
//     Calls whose work overlaps on the GPU (different streams, or different
//     host threads without ordering) race on the array and must be serialised
//     by the caller;
//   * the array's device address belongs to the CUDA context that is current
//     when the call is made (the device's primary context for runtime-API
//     callers, or a context the host pushed itself).  Every call made outside
//     a stream capture looks the address up again with cudaGetSymbolAddress
//     and remembers it for that context; a call whose stream is being captured
//     uses the remembered address, so the first call in a context must come
//     before any stream capture in it.  After cudaDeviceReset the next call
//     outside a capture looks the address up afresh.
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda.h>

#include "../../include/lensdiff_b200.h"
#include "ld_internal.h"

namespace ld {
bool host_factor_plan(int n, bool allow25, FftPlan* plan);
void host_pupil_geometry(PsfBankArgs& a, const ld_params& p);
PhaseCoeffs host_phase_for_wavelength(const ld_params& p, float wavelength);
std::vector<float> host_wavelengths(const ld_params& p);
void host_sizes(const ld_params& p, int* np, int* S, int* R);
}  // namespace ld

using namespace ld;

namespace {

constexpr size_t kNoAllocScratchBytes = 12u << 20;  // 12 MiB
constexpr int kNoAllocMaxPsf = 1024;                // PSF grid S
constexpr int kNoAllocMaxPupil = 512;               // pupil raster N_p
constexpr int kMaxContexts = 64;

// The scratch.  In host code this name is only a host-side stand-in: the
// device address comes from cudaGetSymbolAddress (scratch_address below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Remembered scratch addresses, one per CUDA context.
struct ContextAddress {
    CUcontext ctx;
    unsigned char* addr;
};
std::mutex g_addr_mu;
ContextAddress g_addr[kMaxContexts] = {};
int g_addr_n = 0;

// cuCtxGetCurrent through the runtime's driver entry-point lookup, so the
// library needs no link-time dependency on the driver library.
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
CtxGetCurrentFn ctx_get_current() {
    static CtxGetCurrentFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return static_cast<CtxGetCurrentFn>(nullptr);
        }
        return reinterpret_cast<CtxGetCurrentFn>(f);
    }();
    return fn;
}

// Device address of the scratch in the current context, for work on stream s.
int scratch_address(cudaStream_t s, unsigned char** out, std::string* stage) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        *stage = "no-alloc-no-current-device";
        return LD_ERR_CUDA;
    }
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
        cudaGetLastError();
        cap = cudaStreamCaptureStatusActive;  // unknown: do not call set-up APIs
    }
    void* p = nullptr;
    if (cap == cudaStreamCaptureStatusNone) {
        // also makes the device's primary context current when none is
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            *stage = std::string("no-alloc-symbol-address: ") + cudaGetErrorString(e);
            return LD_ERR_CUDA;
        }
    }
    CtxGetCurrentFn get = ctx_get_current();
    CUcontext ctx = nullptr;
    if (get == nullptr || get(&ctx) != CUDA_SUCCESS || ctx == nullptr) {
        *stage = "no-alloc-no-current-context";
        return LD_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lock(g_addr_mu);
    int slot = -1;
    for (int i = 0; i < g_addr_n; ++i)
        if (g_addr[i].ctx == ctx) slot = i;
    if (cap == cudaStreamCaptureStatusNone) {
        if (slot < 0) {
            if (g_addr_n == kMaxContexts) {
                *stage = "no-alloc-too-many-contexts";
                return LD_ERR_CUDA;
            }
            slot = g_addr_n++;
            g_addr[slot].ctx = ctx;
        }
        g_addr[slot].addr = static_cast<unsigned char*>(p);
    } else if (slot < 0) {
        *stage = "no-alloc-first-call-inside-stream-capture";
        return LD_ERR_ARG;
    }
    *out = g_addr[slot].addr;
    return LD_OK;
}

// tw[k] = exp(-2 pi i k / n), computed in FP64 and stored as float2.
__global__ void noalloc_twiddles(float2* tw, int n) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(-2.0 * static_cast<double>(k) / static_cast<double>(n), &s, &c);
        tw[k] = make_float2(static_cast<float>(c), static_cast<float>(s));
    }
}

// Writes the wavelength constants and clears the energy sum.
__global__ void noalloc_init(WavelengthInfo* wl, WavelengthInfo info, PsfScalars* sc) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        *wl = info;
        *sc = PsfScalars{};
    }
}

size_t align256(size_t n) { return (n + 255) & ~static_cast<size_t>(255); }

void set_stage(ld_status* st, int code, const std::string& s) {
    if (!st) return;
    st->code = code;
    std::strncpy(st->stage, s.c_str(), LD_STAGE_LEN - 1);
    st->stage[LD_STAGE_LEN - 1] = '\0';
}

}  // namespace

extern "C" int ld_raw_psf_noalloc(const ld_params* params, int wavelength_index, float* psf_out, void* stream,
                                  ld_status* st) {
    if (st) std::memset(st, 0, sizeof(*st));
    if (!params || !psf_out) {
        set_stage(st, LD_ERR_ARG, "null-argument");
        return LD_ERR_ARG;
    }
    const ld_params& p = *params;
    if (p.aperture_mode == LD_APERTURE_CUSTOM) {
        set_stage(st, LD_ERR_UNSUPPORTED, "unsupported-custom-aperture");
        return LD_ERR_UNSUPPORTED;
    }
    if (p.aperture_mode < LD_APERTURE_CIRCLE || p.aperture_mode > LD_APERTURE_SNOWFLAKE) {
        set_stage(st, LD_ERR_ARG, "invalid-aperture-mode");
        return LD_ERR_ARG;
    }
    int np = 0, S = 0, R = 0;
    host_sizes(p, &np, &S, &R);
    if (st) {
        st->pupil_size = np;
        st->raw_psf_size = S;
        st->max_kernel_radius = R;
    }
    const std::vector<float> wl = host_wavelengths(p);
    if (wavelength_index < 0 || wavelength_index >= static_cast<int>(wl.size())) {
        set_stage(st, LD_ERR_ARG, "invalid-wavelength-index");
        return LD_ERR_ARG;
    }
    if (S > kNoAllocMaxPsf || np > kNoAllocMaxPupil) {
        set_stage(st, LD_ERR_ARG, "exceeds-no-alloc-limit (pupil <= 512, psf grid <= 1024)");
        return LD_ERR_ARG;
    }
    FftPlan plan{};
    if (!host_factor_plan(S, fft_family(S, 1) == kE25, &plan)) {
        set_stage(st, LD_ERR_UNSUPPORTED, "fft-length-not-5-smooth");
        return LD_ERR_UNSUPPORTED;
    }
    PsfBankArgs a{};
    host_pupil_geometry(a, p);  // pupil parameters, base phase, rows that can be non-zero
    // scratch layout: twiddles | pupil pre-pass | row-pass output | info | sums
    const size_t o_pre = align256(static_cast<size_t>(S) * sizeof(float2));
    const size_t o_rows = o_pre + align256(static_cast<size_t>(np) * np * sizeof(float4));
    const size_t o_wl = o_rows + align256(static_cast<size_t>(a.row_n) * S * sizeof(float2));
    const size_t o_sc = o_wl + align256(sizeof(WavelengthInfo));
    const size_t total = o_sc + align256(sizeof(PsfScalars));
    if (total > kNoAllocScratchBytes) {
        set_stage(st, LD_ERR_ARG, "exceeds-no-alloc-scratch");
        return LD_ERR_ARG;
    }
    // an error left pending by earlier work on this thread is reported as
    // such, not as a failure of these launches
    const cudaError_t pending = cudaGetLastError();
    if (pending != cudaSuccess) {
        set_stage(st, LD_ERR_CUDA, std::string("no-alloc-pending-error-before-call: ") + cudaGetErrorString(pending));
        return LD_ERR_CUDA;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned char* base = nullptr;
    std::string stage;
    const int rc = scratch_address(s, &base, &stage);
    if (rc != LD_OK) {
        set_stage(st, rc, stage);
        return rc;
    }
    float2* tw = reinterpret_cast<float2*>(base);
    plan.tw = tw;
    a.pupil_pre = reinterpret_cast<float4*>(base + o_pre);
    a.rows = reinterpret_cast<float2*>(base + o_rows);
    WavelengthInfo* dwl = reinterpret_cast<WavelengthInfo*>(base + o_wl);
    PsfScalars* dsc = reinterpret_cast<PsfScalars*>(base + o_sc);
    WavelengthInfo wi{};
    wi.phase = host_phase_for_wavelength(p, wl[static_cast<size_t>(wavelength_index)]);
    wi.win_x0 = 0;
    wi.win_n = S;
    a.wl = dwl;
    a.scalars = dsc;
    a.want_energy = 1;
    a.B = 1;
    a.S = S;
    a.half = S / 2;
    a.off = std::max(0, (S - np) / 2);
    a.win_stride = S;
    a.plan_s = plan;
    a.win = psf_out;
    noalloc_twiddles<<<(S + 255) / 256, 256, 0, s>>>(tw, S);
    noalloc_init<<<1, 32, 0, s>>>(dwl, wi, dsc);
    launch_pupil_pre(a, s);
    launch_psf_rows(a, s);
    launch_psf_cols(a, s);
    launch_normalize_psf(psf_out, S * S, dsc, s);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_stage(st, LD_ERR_CUDA, std::string("no-alloc-raw-psf: ") + cudaGetErrorString(e));
        return LD_ERR_CUDA;
    }
    set_stage(st, LD_OK, "ok");
    return LD_OK;
}
