// ld_optics.cuh — per-pixel optics of the LensDiff path, as float32 device code.
//
// Each function restates a reference function with the same float32
// expression order, so that discrete decisions (inside/outside the aperture,
// ring index of a pixel) agree with the reference's CPU code:
//   pupil amplitude  LensDiffCpuReference.cpp:451-488, :670-680, :758-822
//   Zernike phase    LensDiffPhase.cpp:170-243 (Noll 4..17) + standard Noll
//                    j = 1..3, 18..22 (extension)
//   kernel taper     LensDiffCpuReference.cpp:957-982
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace ld {

constexpr float kPiF = 3.14159265358979323846f;
constexpr float kOuterRadius = 0.86f;
constexpr int kMaxVanes = 16;

struct PupilParams {
    int size;          // N_p
    int mode;          // aperture mode (0 circle, 1 polygon, 5 hexagon)
    int sides;         // polygon sides
    int apod;          // apodisation mode
    int vanes;         // vane line count (0: none)
    float roundness;   // clamped to [0,1]
    float rotation;    // radians
    float obstruction; // clamp(obs,0,.95) * outer
    float vane_half;   // thickness * outer
    float decx, decy;  // pupil decenter
    float vane_cs[kMaxVanes];
    float vane_sn[kMaxVanes];
    // phase raster
    float phase_cs, phase_sn;  // cos/sin(-rotation)
};

struct PhaseCoeffs {
    int enabled;       // HasLensDiffNonFlatPhase for this wavelength
    float c[23];       // Noll-indexed float coefficients
};

__device__ __forceinline__ float pupil_coord(int i, int size) {
    return ((static_cast<float>(i) + 0.5f) / static_cast<float>(size) - 0.5f) * 2.0f;
}

// polygonMetric (LensDiffCpuReference.cpp:451-469)
__device__ __forceinline__ float polygon_metric(float nx, float ny, int sides, float roundness, float rotation) {
    const float radius = sqrtf(nx * nx + ny * ny);
    const float circle = radius / fmaxf(kOuterRadius, 1e-5f);
    if (sides < 3) return circle;
    const float angle = atan2f(ny, nx) - rotation;
    const float sector = 2.0f * kPiF / static_cast<float>(sides);
    float local = fmodf(angle, sector);
    if (local < 0.0f) local += sector;
    local -= sector * 0.5f;
    const float poly_r = kOuterRadius * cosf(kPiF / static_cast<float>(sides)) / fmaxf(cosf(local), 1e-4f);
    const float poly = radius / fmaxf(poly_r, 1e-5f);
    return circle * roundness + poly * (1.0f - roundness);
}

// apodizationWeight (LensDiffCpuReference.cpp:670-680)
__device__ __forceinline__ float apodization(int mode, float radial) {
    if (mode == 1) return cosf(fminf(radial, 1.0f) * (kPiF * 0.5f));
    if (mode == 2) return expf(-4.0f * radial * radial);
    return 1.0f;
}

// buildPupilAmplitude per pixel (LensDiffCpuReference.cpp:778-818)
__device__ __forceinline__ float pupil_amplitude(const PupilParams& p, int x, int y) {
    const float nx = pupil_coord(x, p.size);
    const float ny = pupil_coord(y, p.size);
    const float dx = nx - p.decx;
    const float dy = ny - p.decy;
    const float radius = sqrtf(dx * dx + dy * dy);
    bool inside;
    if (p.mode == 0) inside = radius <= kOuterRadius;
    else inside = polygon_metric(dx, dy, p.sides, p.roundness, p.rotation) <= 1.0f;
    if (!inside || radius < p.obstruction) return 0.0f;
    for (int i = 0; i < p.vanes; ++i) {  // blockedByVanes, :471-488
        const float cs = p.vane_cs[i], sn = p.vane_sn[i];
        const float xr = dx * cs + dy * sn;
        const float yr = -dx * sn + dy * cs;
        if (fabsf(yr) <= p.vane_half && fabsf(xr) <= kOuterRadius) return 0.0f;
    }
    return apodization(p.apod, radius / kOuterRadius);
}

// EvaluateLensDiffPhaseWaves + BuildLensDiffPupilPhaseWaves per pixel
// (LensDiffPhase.cpp:170-243).  Returns waves.
__device__ __forceinline__ float pupil_phase(const PupilParams& p, const PhaseCoeffs& c, int x, int y) {
    if (!c.enabled) return 0.0f;
    const float nx = pupil_coord(x, p.size);
    const float ny = pupil_coord(y, p.size);
    const float radius = sqrtf(nx * nx + ny * ny);
    if (radius > kOuterRadius) return 0.0f;
    const float rx = nx * p.phase_cs - ny * p.phase_sn;
    const float ry = nx * p.phase_sn + ny * p.phase_cs;
    const float sx = rx / kOuterRadius - p.decx;
    const float sy = ry / kOuterRadius - p.decy;
    const float r2 = sx * sx + sy * sy;
    if (r2 > 1.0f) return 0.0f;
    const float defocus = 1.7320508075688772f * (2.0f * r2 - 1.0f);
    const float astig0 = 2.4494897427831781f * (sx * sx - sy * sy);
    const float astig45 = 2.4494897427831781f * (2.0f * sx * sy);
    const float comaX = 2.8284271247461901f * ((3.0f * r2 - 2.0f) * sx);
    const float comaY = 2.8284271247461901f * ((3.0f * r2 - 2.0f) * sy);
    const float spherical = 2.2360679774997898f * (6.0f * r2 * r2 - 6.0f * r2 + 1.0f);
    const float trefoilX = 2.8284271247461901f * (sx * sx * sx - 3.0f * sx * sy * sy);
    const float trefoilY = 2.8284271247461901f * (3.0f * sx * sx * sy - sy * sy * sy);
    const float sar = 4.0f * r2 - 3.0f;
    const float sa0 = 3.1622776601683795f * sar * (sx * sx - sy * sy);
    const float sa45 = 3.1622776601683795f * sar * (2.0f * sx * sy);
    const float q0 = 3.1622776601683795f * (sx * sx * sx * sx - 6.0f * sx * sx * sy * sy + sy * sy * sy * sy);
    const float q45 = 3.1622776601683795f * (4.0f * sx * sy * (sx * sx - sy * sy));
    const float scr = 10.0f * r2 * r2 - 12.0f * r2 + 3.0f;
    const float scX = 3.4641016151377544f * scr * sx;
    const float scY = 3.4641016151377544f * scr * sy;
    float v = c.c[4] * defocus + c.c[6] * astig0 + c.c[5] * astig45 + c.c[8] * comaX + c.c[7] * comaY +
              c.c[11] * spherical + c.c[10] * trefoilX + c.c[9] * trefoilY + c.c[12] * sa0 + c.c[13] * sa45 +
              c.c[14] * q0 + c.c[15] * q45 + c.c[16] * scX + c.c[17] * scY;
    // extension terms: standard Noll (even j: cos m*theta, odd j: sin m*theta)
    const float x2 = sx * sx, y2 = sy * sy;
    v += c.c[1] + c.c[2] * (2.0f * sx) + c.c[3] * (2.0f * sy);
    const float r3rad = 5.0f * r2 - 4.0f;
    v += c.c[18] * (3.4641016151377544f * r3rad * (sx * (x2 - 3.0f * y2)));
    v += c.c[19] * (3.4641016151377544f * r3rad * (sy * (3.0f * x2 - y2)));
    v += c.c[20] * (3.4641016151377544f * (sx * (x2 * x2 - 10.0f * x2 * y2 + 5.0f * y2 * y2)));
    v += c.c[21] * (3.4641016151377544f * (sy * (5.0f * x2 * x2 - 10.0f * x2 * y2 + y2 * y2)));
    v += c.c[22] * (2.6457513110645906f * (20.0f * r2 * r2 * r2 - 30.0f * r2 * r2 + 12.0f * r2 - 1.0f));
    return v;
}

// The phase of one pupil pixel split as phi = phi0 + c4 * z4: phi0 collects
// every term but defocus, z4 is the defocus polynomial.  Only defocus varies
// across the wavelengths of a bank (the chromatic focus offset,
// LensDiffCpuReference.cpp:1721-1723), so phi0 and z4 are computed once per
// bank.  `valid` is 0 outside the phase support (radius > outer or r^2 > 1).
__device__ __forceinline__ void pupil_phase_split(const PupilParams& p, const PhaseCoeffs& c, int x, int y,
                                                  float* phi0, float* z4, float* valid) {
    PhaseCoeffs c0 = c;
    c0.enabled = 1;
    const float c4 = c0.c[4];
    c0.c[4] = 0.0f;
    *phi0 = pupil_phase(p, c0, x, y);
    c0 = PhaseCoeffs{};
    c0.enabled = 1;
    c0.c[4] = 1.0f;
    *z4 = pupil_phase(p, c0, x, y);
    (void)c4;
    // the support test of pupil_phase, repeated
    const float nx = pupil_coord(x, p.size);
    const float ny = pupil_coord(y, p.size);
    const float radius = sqrtf(nx * nx + ny * ny);
    bool ok = radius <= kOuterRadius;
    if (ok) {
        const float rx = nx * p.phase_cs - ny * p.phase_sn;
        const float ry = nx * p.phase_sn + ny * p.phase_cs;
        const float sx = rx / kOuterRadius - p.decx;
        const float sy = ry / kOuterRadius - p.decy;
        ok = sx * sx + sy * sy <= 1.0f;
    }
    *valid = ok ? 1.0f : 0.0f;
}

// Pupil field sample A * exp(i 2 pi phi) (LensDiffCpuReference.cpp:838-848).
__device__ __forceinline__ float2 pupil_field(const PupilParams& p, const PhaseCoeffs& c, int x, int y) {
    const float a = pupil_amplitude(p, x, y);
    if (a <= 0.0f) return make_float2(a, 0.0f);
    const float ph = pupil_phase(p, c, x, y);
    if (ph == 0.0f) return make_float2(a, 0.0f);
    float sn, cs;
    sincosf(ph * 2.0f * kPiF, &sn, &cs);
    return make_float2(a * cs, a * sn);
}

// applySupportBoundaryTaper weight (LensDiffCpuReference.cpp:962-978);
// extent/fade/start precomputed per kernel.
__device__ __forceinline__ float taper_weight(float radius, float extent, float fade, float start) {
    if (radius >= extent) return 0.0f;
    const float t = fminf(fmaxf((radius - start) / fmaxf(fade, 1e-6f), 0.0f), 1.0f);
    const float s = t * t * (3.0f - 2.0f * t);
    return fmaxf(0.0f, cosf(s * static_cast<float>(3.14159265358979323846 * 0.5)));
}

}  // namespace ld
