// ref_shim.cpp — TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// Builds the reference's own CPU implementation of the LensDiff path from its
// sources where they lie (the Makefile in this folder points the include path
// at the reference tree; nothing is copied) and exposes it to the tests
// through a small extern "C" surface.  The reference translation unit
// source/src/core/LensDiffCpuReference.cpp is #included here so that its
// file-static stages (convolveScalar, buildSelectionMask, ...) can be timed
// and compared one by one; the other five CPU sources are linked normally.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
// the resulting oracle/_ref/libldref.so.

#include "LensDiffCpuReference.cpp"  // reference TU, compiled in place
// and its aperture-image loader, in place too, so the checker can seed the
// loader's own cache with an image decoded here (the loader's decoders are
// WIC / ImageIO only)
#include "LensDiffApertureImage.cpp"

#include "lensdiff_b200.h"
#include "ref_params.h"

#include <cstring>

namespace {

void copyStage(const std::string& s, char* out, int cap) {
    if (out == nullptr || cap <= 0) return;
    std::strncpy(out, s.c_str(), static_cast<std::size_t>(cap - 1));
    out[cap - 1] = '\0';
}

}  // namespace

extern "C" {

// Puts a decoded amplitude image (h rows of w floats) into the reference's
// aperture-image cache (LensDiffApertureImage.cpp:301-365) under a path that
// names no file, so LoadLensDiffPreparedApertureImage finds it there and
// applies its own normalise / invert; Custom-mode calls then use it.
void ldref_set_custom_aperture(const float* values, int w, int h, int normalize, int invert) {
    const std::string path = "lensdiff-b200-checker-decoded-aperture";
    LensDiffApertureImage img;
    img.width = w;
    img.height = h;
    img.values.assign(values, values + static_cast<std::size_t>(w) * h);
    {
        std::lock_guard<std::mutex> lock(apertureImageCacheMutex());
        CachedApertureImage& cached = apertureImageCache()[path];
        cached.hasTimestamp = false;
        cached.image = img;
    }
    refCustomAperture().path = path;
    refCustomAperture().normalize = normalize != 0;
    refCustomAperture().invert = invert != 0;
}

// Path sizes: N_p, S, R_max (LensDiffCpuReference.cpp:1709-1711).
void ldref_sizes(const ld_params* p, int* pupil, int* raw, int* rmax) {
    const LensDiffParams r = toReference(*p);
    const int np = GetLensDiffEffectivePupilResolution(r.pupilResolution);
    const int rm = std::max(4, ResolveLensDiffMaxKernelRadiusPx(r));
    *pupil = np;
    *rmax = rm;
    *raw = ChooseLensDiffRawPsfSize(np, rm);
}

// Pupil amplitude and phase (waves), N_p^2 each (CpuReference.cpp:758-829).
void ldref_pupil(const ld_params* p, float* amp, float* phase) {
    const LensDiffParams r = toReference(*p);
    const std::vector<float> a = BuildLensDiffPupilAmplitudeForPsf(r);
    const std::vector<float> f = BuildLensDiffPupilPhaseForPsf(r);
    std::memcpy(amp, a.data(), a.size() * sizeof(float));
    std::memcpy(phase, f.data(), f.size() * sizeof(float));
}

// Shifted, normalised raw PSF (S^2) for the given wavelength, with the
// chromatic-focus defocus offset applied as buildPsfBankGlobalOnly does
// (CpuReference.cpp:1720-1728).
void ldref_raw_psf(const ld_params* p, float wavelength, float* out) {
    LensDiffParams r = toReference(*p);
    const int np = GetLensDiffEffectivePupilResolution(r.pupilResolution);
    const int rm = std::max(4, ResolveLensDiffMaxKernelRadiusPx(r));
    const int s = ChooseLensDiffRawPsfSize(np, rm);
    const std::vector<float> pupil = BuildLensDiffPupilAmplitudeForPsf(r);
    const float wavelengthOffset = (wavelength - 550.0f) / 110.0f;
    r.phaseDefocus += r.chromaticFocus * wavelengthOffset;
    if (std::abs(r.phaseDefocus) > 1e-6) r.phaseMode = LensDiffPhaseMode::Enabled;
    const std::vector<float> phase = BuildLensDiffPupilPhaseForPsf(r);
    const std::vector<float> raw = BuildLensDiffShiftedRawPsf(pupil, phase, np, s);
    std::memcpy(out, raw.data(), raw.size() * sizeof(float));
}

// First-minimum radius of the clear-circle reference PSF (CpuReference.cpp:2018-2038, :897-955).
float ldref_first_zero(int pupil, int raw) {
    auto ref = GetLensDiffReferenceRawPsfCached(pupil, raw);
    return EstimateLensDiffFirstMinimumRadius(*ref, raw);
}

float ldref_first_zero_of(const float* psf, int size) {
    std::vector<float> v(psf, psf + static_cast<std::size_t>(size) * size);
    return EstimateLensDiffFirstMinimumRadius(v, size);
}

// Wavelengths of the reference spectral mode (CpuReference.cpp:1602-1614).
int ldref_wavelengths(int mode, float* out) {
    const std::vector<float> w = GetLensDiffSpectralWavelengths(static_cast<LensDiffSpectralMode>(mode));
    for (std::size_t i = 0; i < w.size(); ++i) out[i] = w[i];
    return static_cast<int>(w.size());
}

// PSF bank: for every bin the full / core / structure kernels
// (EnsureLensDiffPsfBank, CpuReference.cpp:2068).  Kernels are written
// back-to-back; sizes[i] is the side of bin i.  Returns the bin count, or -1
// when capacity is too small.  Field zones are not exported.
int ldref_bank(const ld_params* p, float* wavelengths, int* sizes, float* full, float* core,
               float* structure, long long capacity, int* support_radius) {
    const LensDiffParams r = toReference(*p);
    LensDiffPsfBankCache cache {};
    EnsureLensDiffPsfBank(r, cache);
    long long off = 0;
    for (std::size_t i = 0; i < cache.bins.size(); ++i) {
        const auto& b = cache.bins[i];
        const long long n = static_cast<long long>(b.full.values.size());
        if (off + n > capacity) return -1;
        wavelengths[i] = b.wavelengthNm;
        sizes[i] = b.full.size;
        std::memcpy(full + off, b.full.values.data(), n * sizeof(float));
        if (core) std::memcpy(core + off, b.core.values.data(), n * sizeof(float));
        if (structure) std::memcpy(structure + off, b.structure.values.data(), n * sizeof(float));
        off += n;
    }
    if (support_radius) *support_radius = cache.supportRadiusPx;
    return static_cast<int>(cache.bins.size());
}

// Spectrum configuration for the given wavelengths (LensDiffSpectrum.cpp:380-460):
// natural and style matrices, row-major 3 x 9 as in LensDiffSpectrumConfig.
int ldref_spectrum_config(const ld_params* p, int count, const float* wavelengths,
                          float* natural27, float* style27) {
    const LensDiffParams r = toReference(*p);
    std::vector<LensDiffPsfBin> bins(static_cast<std::size_t>(count));
    for (int i = 0; i < count; ++i) bins[static_cast<std::size_t>(i)].wavelengthNm = wavelengths[i];
    const LensDiffSpectrumConfig c = BuildLensDiffSpectrumConfig(r, bins);
    std::memcpy(natural27, c.naturalMatrix.data(), 27 * sizeof(float));
    std::memcpy(style27, c.styleMatrix.data(), 27 * sizeof(float));
    return c.binCount;
}

// MapLensDiffSpectralBins over n pixels (LensDiffSpectrum.cpp:462-497);
// values is n x 9, rgb_out n x 3.
void ldref_map_bins(const ld_params* p, int count, const float* wavelengths, const float* values,
                    long long n, float* rgb_out) {
    const LensDiffParams r = toReference(*p);
    std::vector<LensDiffPsfBin> bins(static_cast<std::size_t>(count));
    for (int i = 0; i < count; ++i) bins[static_cast<std::size_t>(i)].wavelengthNm = wavelengths[i];
    const LensDiffSpectrumConfig c = BuildLensDiffSpectrumConfig(r, bins);
    for (long long k = 0; k < n; ++k) {
        std::array<float, kLensDiffMaxSpectralBins> v {};
        for (int i = 0; i < kLensDiffMaxSpectralBins; ++i) v[static_cast<std::size_t>(i)] = values[k * 9 + i];
        const auto rgb = MapLensDiffSpectralBins(v, r, c);
        rgb_out[k * 3 + 0] = rgb[0];
        rgb_out[k * 3 + 1] = rgb[1];
        rgb_out[k * 3 + 2] = rgb[2];
    }
}

// Full CPU render (RunLensDiffCpuReference, CpuReference.cpp:2073-2261) on
// HOST float RGBA images.  src is width x height at bounds origin (sx1, sy1);
// dst has its own bounds; render window given explicitly.
int ldref_render(const ld_params* p, const float* src, int sx1, int sy1, int sw, int sh,
                 float* dst, int dx1, int dy1, int dw, int dh,
                 int rx1, int ry1, int rx2, int ry2, char* error, int error_cap) {
    const LensDiffParams r = toReference(*p);
    LensDiffRenderRequest req {};
    req.renderWindow = {rx1, ry1, rx2, ry2};
    req.frameBounds = {sx1, sy1, sx1 + sw, sy1 + sh};
    req.src.data = const_cast<float*>(src);
    req.src.rowBytes = static_cast<std::ptrdiff_t>(sw) * 16;
    req.src.bounds = {sx1, sy1, sx1 + sw, sy1 + sh};
    req.dst.data = dst;
    req.dst.rowBytes = static_cast<std::ptrdiff_t>(dw) * 16;
    req.dst.bounds = {dx1, dy1, dx1 + dw, dy1 + dh};
    req.frameShortSidePx = r.frameShortSidePx;
    LensDiffPsfBankCache cache {};
    std::string err;
    const bool ok = RunLensDiffCpuReference(req, r, cache, &err);
    copyStage(err, error, error_cap);
    return ok ? 1 : 0;
}

// One reference bin convolution (convolveScalar, CpuReference.cpp:1167-1193):
// src width x height, square odd kernel of side ksize.  Used to time the
// reference's per-bin cost.
void ldref_convolve_scalar(const float* src, int width, int height, const float* kernel, int ksize,
                           float* out) {
    ScalarImage img(width, height);
    std::memcpy(img.pixels.data(), src, static_cast<std::size_t>(width) * height * sizeof(float));
    LensDiffKernel k {};
    k.size = ksize;
    k.values.assign(kernel, kernel + static_cast<std::size_t>(ksize) * ksize);
    const ScalarImage o = convolveScalar(img, k);
    std::memcpy(out, o.pixels.data(), o.pixels.size() * sizeof(float));
}

// Reference raw PSF from explicit pupil / phase rasters (BuildLensDiffShiftedRawPsf).
void ldref_raw_psf_from(const float* pupil, const float* phase, int np, int s, float* out) {
    std::vector<float> a(pupil, pupil + static_cast<std::size_t>(np) * np);
    std::vector<float> f;
    if (phase) f.assign(phase, phase + static_cast<std::size_t>(np) * np);
    const std::vector<float> raw = BuildLensDiffShiftedRawPsf(a, f, np, s);
    std::memcpy(out, raw.data(), raw.size() * sizeof(float));
}

// Resampled base kernel (makeResampledKernel, CpuReference.cpp:1060-1086).
void ldref_resample(const float* raw, int s, float scale, int radius, float* out) {
    std::vector<float> v(raw, raw + static_cast<std::size_t>(s) * s);
    const LensDiffKernel k = makeResampledKernel(v, s, scale, radius);
    std::memcpy(out, k.values.data(), k.values.size() * sizeof(float));
}

}  // extern "C"
