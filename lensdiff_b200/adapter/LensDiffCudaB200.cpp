// LensDiffCudaB200.cpp — drop-in replacement of the plugin's CUDA backend call.
//
// Compiled inside the LensDiff plugin tree in place of
// source/src/cuda/LensDiffCuda.cu, against the plugin's own headers
// (LensDiffTypes.h, LensDiffSpectrum.h), and linked with liblensdiff_b200.so.
// It keeps the exact entry point the plugin calls at LensDiff.cpp:3833:
//
//     bool RunLensDiffCuda(const LensDiffRenderRequest& request,
//                          const LensDiffParams& params,
//                          LensDiffPsfBankCache& cache,
//                          std::string* error);        // LensDiffCuda.h:7-10
//
// and maps its arguments field by field onto the C ABI of
// include/lensdiff_b200.h.  The spectral->RGB matrices come from the plugin's
// own BuildLensDiffSpectrumConfig (LensDiffSpectrum.cpp:380-460), exactly as
// the reference CUDA backend obtains them (LensDiffCuda.cu:4779).  Errors are
// returned as `false` plus the library's stage string; there is no CPU
// fallback, as in the reference (LensDiff.cpp:3822-3823).
//
// One library context per CUDA device serves every effect instance; the
// device-resident PSF-bank cache lives in that context (the plugin's
// LensDiffPsfBankCache is left untouched unless a caller needs host kernels).
//
// Environment switches, read once per process in the style of the reference
// backend's LENSDIFF_CUDA_* variables (LensDiffCuda.cu:462-517):
//   LENSDIFF_B200_FFT_FORM       chosen (default): tensor-core PSF windows and
//                                FP16 frame spectra; fp32: the hand-written FP32
//                                chain; cufft: the cuFFT comparator chain.
//   LENSDIFF_B200_HBM_BUDGET_MB  device memory the library context may hold
//                                (0 or unset: no budget).
#include "LensDiffSpectrum.h"
#include "LensDiffTypes.h"
#include "lensdiff_b200.h"

#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace {

// LENSDIFF_B200_FFT_FORM; an unknown value selects the default form.
int32_t fftFormFromEnvironment() {
    static const int32_t form = [] {
        const char* v = std::getenv("LENSDIFF_B200_FFT_FORM");
        if (v != nullptr && std::strcmp(v, "fp32") == 0) return static_cast<int32_t>(LD_FFT_OWN_FP32);
        if (v != nullptr && std::strcmp(v, "cufft") == 0) return static_cast<int32_t>(LD_FFT_CUFFT);
        return static_cast<int32_t>(LD_FFT_OWN_CHOSEN);
    }();
    return form;
}

std::size_t hbmBudgetFromEnvironment() {
    const char* v = std::getenv("LENSDIFF_B200_HBM_BUDGET_MB");
    if (v == nullptr) return 0;
    const long long mb = std::atoll(v);
    return mb > 0 ? static_cast<std::size_t>(mb) << 20 : 0;
}

std::mutex& contextMutex() {
    static std::mutex m;
    return m;
}

ld_ctx* contextForCurrentDevice(std::string* error) {
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        if (error) *error = "cuda-get-device-failed";
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(contextMutex());
    static std::map<int, ld_ctx*> contexts;
    auto it = contexts.find(device);
    if (it != contexts.end()) return it->second;
    ld_ctx* ctx = nullptr;
    if (ld_create(&ctx, device, hbmBudgetFromEnvironment()) != LD_OK) {
        if (error) *error = "lensdiff-b200-context-create-failed";
        return nullptr;
    }
    contexts[device] = ctx;
    return ctx;
}

ld_rect toRect(const LensDiffImageRect& r) { return ld_rect{r.x1, r.y1, r.x2, r.y2}; }

ld_image_view toView(const LensDiffImageView& v) {
    ld_image_view out{};
    out.data = v.data;
    out.row_bytes = static_cast<int64_t>(v.rowBytes);
    out.bounds = toRect(v.bounds);
    out.origin_x = v.originX;
    out.origin_y = v.originY;
    out.components = v.components;
    out.bytes_per_component = v.bytesPerComponent;
    return out;
}

// LensDiffParams (LensDiffTypes.h:128-208) -> ld_params.
ld_params toParams(const LensDiffParams& p) {
    ld_params o;
    std::memset(&o, 0, sizeof(o));
    o.extraction_mode = static_cast<int32_t>(p.extractionMode);
    o.aperture_mode = static_cast<int32_t>(p.apertureMode);
    o.apodization_mode = static_cast<int32_t>(p.apodizationMode);
    o.spectral_mode = static_cast<int32_t>(p.spectralMode);
    o.spectrum_style = static_cast<int32_t>(p.spectrumStyle);
    o.look_mode = static_cast<int32_t>(p.lookMode);
    o.energy_mode = static_cast<int32_t>(p.energyMode);
    o.debug_view = static_cast<int32_t>(p.debugView);
    o.input_transfer = static_cast<int32_t>(p.inputTransfer);
    o.resolution_aware = p.resolutionAware ? 1 : 0;
    o.threshold = p.threshold;
    o.softness_stops = p.softnessStops;
    o.point_emphasis = p.pointEmphasis;
    o.core_preserve = p.corePreserve;
    o.blade_count = p.bladeCount;
    o.vane_count = p.vaneCount;
    o.roundness = p.roundness;
    o.rotation_deg = p.rotationDeg;
    o.central_obstruction = p.centralObstruction;
    o.vane_thickness = p.vaneThickness;
    o.diffraction_scale_px = p.diffractionScalePx;
    o.pupil_resolution = p.pupilResolution;
    o.frame_short_side_px = p.frameShortSidePx;
    o.max_kernel_radius_px = p.maxKernelRadiusPx;
    o.phase_mode = static_cast<int32_t>(p.phaseMode);
    o.chromatic_affects_luma = p.chromaticAffectsLuma ? 1 : 0;
    o.phase_defocus = p.phaseDefocus;
    o.phase_astigmatism0 = p.phaseAstigmatism0;
    o.phase_astigmatism45 = p.phaseAstigmatism45;
    o.phase_coma_x = p.phaseComaX;
    o.phase_coma_y = p.phaseComaY;
    o.phase_spherical = p.phaseSpherical;
    o.phase_trefoil_x = p.phaseTrefoilX;
    o.phase_trefoil_y = p.phaseTrefoilY;
    o.phase_secondary_astigmatism0 = p.phaseSecondaryAstigmatism0;
    o.phase_secondary_astigmatism45 = p.phaseSecondaryAstigmatism45;
    o.phase_quadrafoil0 = p.phaseQuadrafoil0;
    o.phase_quadrafoil45 = p.phaseQuadrafoil45;
    o.phase_secondary_coma_x = p.phaseSecondaryComaX;
    o.phase_secondary_coma_y = p.phaseSecondaryComaY;
    o.pupil_decenter_x = p.pupilDecenterX;
    o.pupil_decenter_y = p.pupilDecenterY;
    o.phase_field_strength = p.phaseFieldStrength;
    o.phase_field_edge_bias = p.phaseFieldEdgeBias;
    o.phase_field_defocus = p.phaseFieldDefocus;
    o.phase_field_astig_radial = p.phaseFieldAstigRadial;
    o.phase_field_astig_tangential = p.phaseFieldAstigTangential;
    o.phase_field_coma_radial = p.phaseFieldComaRadial;
    o.phase_field_coma_tangential = p.phaseFieldComaTangential;
    o.phase_field_spherical = p.phaseFieldSpherical;
    o.phase_field_trefoil_radial = p.phaseFieldTrefoilRadial;
    o.phase_field_trefoil_tangential = p.phaseFieldTrefoilTangential;
    o.phase_field_secondary_astig_radial = p.phaseFieldSecondaryAstigRadial;
    o.phase_field_secondary_astig_tangential = p.phaseFieldSecondaryAstigTangential;
    o.phase_field_quadrafoil_radial = p.phaseFieldQuadrafoilRadial;
    o.phase_field_quadrafoil_tangential = p.phaseFieldQuadrafoilTangential;
    o.phase_field_secondary_coma_radial = p.phaseFieldSecondaryComaRadial;
    o.phase_field_secondary_coma_tangential = p.phaseFieldSecondaryComaTangential;
    o.spectrum_force = p.spectrumForce;
    o.spectrum_saturation = p.spectrumSaturation;
    o.chromatic_focus = p.chromaticFocus;
    o.chromatic_spread = p.chromaticSpread;
    o.creative_fringe = p.creativeFringe;
    o.scatter_amount = p.scatterAmount;
    o.scatter_radius = p.scatterRadius;
    o.effect_gain = p.effectGain;
    o.core_compensation = p.coreCompensation;
    o.anisotropy_emphasis = p.anisotropyEmphasis;
    o.core_gain = p.coreGain;
    o.structure_gain = p.structureGain;
    o.core_shoulder = p.coreShoulder;
    o.structure_shoulder = p.structureShoulder;
    o.rgb_mode = LD_RGB_FROM_CALLER;
    o.fft_form = fftFormFromEnvironment();
    return o;
}

// Spectral matrices of the mode's wavelengths from the plugin's own
// BuildLensDiffSpectrumConfig (row-major 3 x 9 in the config, 3 x B here).
void fillSpectrumMatrices(const LensDiffParams& params, ld_params* out) {
    if (params.spectralMode == LensDiffSpectralMode::Mono) return;
    static const float kTri[] = {460.0f, 550.0f, 610.0f};
    static const float k5[] = {440.0f, 490.0f, 540.0f, 590.0f, 640.0f};
    static const float k9[] = {420.0f, 450.0f, 480.0f, 510.0f, 540.0f, 570.0f, 600.0f, 630.0f, 660.0f};
    const float* wl = kTri;
    int count = 3;
    if (params.spectralMode == LensDiffSpectralMode::Spectral5) {
        wl = k5;
        count = 5;
    } else if (params.spectralMode == LensDiffSpectralMode::Spectral9) {
        wl = k9;
        count = 9;
    }
    std::vector<LensDiffPsfBin> bins(static_cast<std::size_t>(count));
    for (int i = 0; i < count; ++i) bins[static_cast<std::size_t>(i)].wavelengthNm = wl[i];
    const LensDiffSpectrumConfig cfg = BuildLensDiffSpectrumConfig(params, bins);
    for (int c = 0; c < 3; ++c) {
        for (int b = 0; b < count; ++b) {
            out->natural_matrix[c * count + b] = cfg.naturalMatrix[static_cast<std::size_t>(c * kLensDiffMaxSpectralBins + b)];
            out->style_matrix[c * count + b] = cfg.styleMatrix[static_cast<std::size_t>(c * kLensDiffMaxSpectralBins + b)];
        }
    }
}

}  // namespace

bool RunLensDiffCuda(const LensDiffRenderRequest& request,
                     const LensDiffParams& params,
                     LensDiffPsfBankCache& cache,
                     std::string* error) {
    (void)cache;  // the bank is cached on the device by the library context
    ld_ctx* ctx = contextForCurrentDevice(error);
    if (ctx == nullptr) return false;
    ld_render_request rq{};
    rq.render_window = toRect(request.renderWindow);
    rq.frame_bounds = toRect(request.frameBounds);
    rq.src = toView(request.src);
    rq.dst = toView(request.dst);
    rq.frame_short_side_px = request.frameShortSidePx;
    rq.host_enabled_cuda_render = request.hostEnabledCudaRender ? 1 : 0;
    rq.cuda_stream = request.cudaStream;
    ld_params p = toParams(params);
    fillSpectrumMatrices(params, &p);
    ld_status st{};
    const int rc = ld_render(ctx, &rq, &p, &st);
    if (rc != LD_OK) {
        if (error) *error = st.stage;
        return false;
    }
    return true;
}
