// ld_optics.cuh — per-pixel optics of the LensDiff path, as float32 device code.
//
// Each function restates a reference function with the same float32
// expression order, so that discrete decisions (inside/outside the aperture,
// ring index of a pixel) agree with the reference's CPU code:
//   pupil amplitude  LensDiffCpuReference.cpp:451-488, :509-668, :670-680, :758-822
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
    int mode;          // aperture mode (LD_APERTURE_*; hexagon is a 6-sided polygon)
    int sides;         // polygon sides / star points / grid divisions / spiral arms (>= 3)
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
    // per-mode constants, computed on the host with the reference's float
    // expressions (they are the same for every pixel)
    float star_inner;          // Star: inner radius (outer * clamped inner ratio)
    float spiral_twist, spiral_opening;
    float grid_half, grid_pitch, grid_bar;  // SquareGrid
    int snow_levels;                        // Snowflake
    float snow_main, snow_thick;
    float snow_arm_cs[6], snow_arm_sn[6];
    float snow_br_cs[6][2], snow_br_sn[6][2];
    float snow_t[5], snow_len[5];
    // Custom: the prepared amplitude image (device, ch rows of cw) and its
    // fit inside the unit square (buildCustomPupilAmplitude's fitHalfWidth /
    // fitHalfHeight); null for the other modes
    const float* custom;
    int cw, ch;
    float fit_hw, fit_hh;
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

// starMetric (LensDiffCpuReference.cpp:509-536)
__device__ __forceinline__ float star_metric(float nx, float ny, int points, float inner, float rotation) {
    const float radius = sqrtf(nx * nx + ny * ny);
    if (radius <= 1e-6f) return 0.0f;
    const float angle = atan2f(ny, nx) - rotation + kPiF * 0.5f;
    const float sector = 2.0f * kPiF / static_cast<float>(points);
    float local = fmodf(angle, sector);
    if (local < 0.0f) local += sector;
    const float half = sector * 0.5f;
    const float t = local <= half ? local / fmaxf(half, 1e-6f) : (sector - local) / fmaxf(half, 1e-6f);
    const float boundary = inner + (kOuterRadius - inner) * fminf(fmaxf(t, 0.0f), 1.0f);
    return radius / fmaxf(boundary, 1e-5f);
}

// distancePointToSegment (LensDiffCpuReference.cpp:558-574)
__device__ __forceinline__ float segment_distance(float px, float py, float ax, float ay, float bx, float by) {
    const float vx = bx - ax;
    const float vy = by - ay;
    const float len2 = vx * vx + vy * vy;
    if (len2 <= 1e-10f) {
        const float dx = px - ax;
        const float dy = py - ay;
        return sqrtf(dx * dx + dy * dy);
    }
    const float t = fminf(fmaxf(((px - ax) * vx + (py - ay) * vy) / len2, 0.0f), 1.0f);
    const float cx = ax + t * vx;
    const float cy = ay + t * vy;
    const float dx = px - cx;
    const float dy = py - cy;
    return sqrtf(dx * dx + dy * dy);
}

// squareGridMaskOpen (LensDiffCpuReference.cpp:576-606)
__device__ __forceinline__ bool square_grid_open(const PupilParams& p, float nx, float ny) {
    const float rx = nx * p.phase_cs - ny * p.phase_sn;
    const float ry = nx * p.phase_sn + ny * p.phase_cs;
    const float h = p.grid_half;
    if (fabsf(rx) > h || fabsf(ry) > h) return false;
    auto nearest = [&](float v) {
        const float wrapped = fmodf(v + h, p.grid_pitch);
        const float positive = wrapped < 0.0f ? wrapped + p.grid_pitch : wrapped;
        return fminf(positive, p.grid_pitch - positive);
    };
    const float dx = nearest(rx), dy = nearest(ry);
    const float ex = fabsf(fabsf(rx) - h), ey = fabsf(fabsf(ry) - h);
    return dx <= p.grid_bar || dy <= p.grid_bar || ex <= p.grid_bar || ey <= p.grid_bar;
}

// snowflakeMaskOpen (LensDiffCpuReference.cpp:608-648)
__device__ __forceinline__ bool snowflake_open(const PupilParams& p, float nx, float ny) {
    const float radius = sqrtf(nx * nx + ny * ny);
    if (radius > kOuterRadius) return false;
    float best = 3.402823466e38f;
    for (int arm = 0; arm < 6; ++arm) {
        const float cs = p.snow_arm_cs[arm], sn = p.snow_arm_sn[arm];
        best = fminf(best, segment_distance(nx, ny, 0.0f, 0.0f, cs * p.snow_main, sn * p.snow_main));
        for (int level = 0; level < p.snow_levels; ++level) {
            const float t = p.snow_t[level];
            const float mx = cs * p.snow_main * t;
            const float my = sn * p.snow_main * t;
            for (int side = 0; side < 2; ++side) {
                const float bx = mx + p.snow_br_cs[arm][side] * p.snow_len[level];
                const float by = my + p.snow_br_sn[arm][side] * p.snow_len[level];
                best = fminf(best, segment_distance(nx, ny, mx, my, bx, by));
            }
        }
    }
    return best <= p.snow_thick;
}

// spiralMaskOpen (LensDiffCpuReference.cpp:650-668)
__device__ __forceinline__ bool spiral_open(const PupilParams& p, float nx, float ny) {
    const float radius = sqrtf(nx * nx + ny * ny);
    if (radius > kOuterRadius) return false;
    const float radial = radius / fmaxf(kOuterRadius, 1e-6f);
    const float angle = atan2f(ny, nx) - p.rotation;
    const float phase = static_cast<float>(p.sides) * angle + p.spiral_twist * radial * (2.0f * kPiF);
    const float band = 0.5f + 0.5f * cosf(phase);
    return band >= (1.0f - p.spiral_opening);
}

// buildPupilAmplitude per pixel (LensDiffCpuReference.cpp:778-818)
// sampleImageBilinear (LensDiffCpuReference.cpp:682-705) on the custom image.
__device__ __forceinline__ float custom_sample(const PupilParams& p, float x, float y) {
    if (x < 0.0f || y < 0.0f || x > static_cast<float>(p.cw - 1) || y > static_cast<float>(p.ch - 1)) return 0.0f;
    const int x0 = static_cast<int>(floorf(x));
    const int y0 = static_cast<int>(floorf(y));
    const int x1 = min(x0 + 1, p.cw - 1);
    const int y1 = min(y0 + 1, p.ch - 1);
    const float tx = __fsub_rn(x, static_cast<float>(x0));
    const float ty = __fsub_rn(y, static_cast<float>(y0));
    const float v00 = __ldg(p.custom + static_cast<size_t>(y0) * p.cw + x0);
    const float v10 = __ldg(p.custom + static_cast<size_t>(y0) * p.cw + x1);
    const float v01 = __ldg(p.custom + static_cast<size_t>(y1) * p.cw + x0);
    const float v11 = __ldg(p.custom + static_cast<size_t>(y1) * p.cw + x1);
    const float vx0 = __fadd_rn(v00, __fmul_rn(__fsub_rn(v10, v00), tx));
    const float vx1 = __fadd_rn(v01, __fmul_rn(__fsub_rn(v11, v01), tx));
    return __fadd_rn(vx0, __fmul_rn(__fsub_rn(vx1, vx0), ty));
}

// buildCustomPupilAmplitude per pixel (LensDiffCpuReference.cpp:707-756): the
// image, rotated with the aperture and fitted into the outer circle, times
// the apodisation; no obstruction or vanes.  Unfused float operations, as the
// reference evaluates them, so the fit and range decisions agree.
__device__ __forceinline__ float custom_amplitude(const PupilParams& p, float dx, float dy) {
    const float radius = sqrtf(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
    if (radius > kOuterRadius || p.custom == nullptr) return 0.0f;
    const float rx = __fsub_rn(__fmul_rn(dx, p.phase_cs), __fmul_rn(dy, p.phase_sn));
    const float ry = __fadd_rn(__fmul_rn(dx, p.phase_sn), __fmul_rn(dy, p.phase_cs));
    const float ux = __fdiv_rn(rx, kOuterRadius);
    const float uy = __fdiv_rn(ry, kOuterRadius);
    if (fabsf(ux) > p.fit_hw || fabsf(uy) > p.fit_hh) return 0.0f;
    const float sx = __fmul_rn(__fadd_rn(__fmul_rn(__fdiv_rn(ux, p.fit_hw), 0.5f), 0.5f), static_cast<float>(p.cw - 1));
    const float sy = __fmul_rn(__fadd_rn(__fmul_rn(__fdiv_rn(uy, p.fit_hh), 0.5f), 0.5f), static_cast<float>(p.ch - 1));
    return __fmul_rn(custom_sample(p, sx, sy), apodization(p.apod, __fdiv_rn(radius, kOuterRadius)));
}

__device__ __forceinline__ float pupil_amplitude(const PupilParams& p, int x, int y) {
    const float nx = pupil_coord(x, p.size);
    const float ny = pupil_coord(y, p.size);
    const float dx = nx - p.decx;
    const float dy = ny - p.decy;
    if (p.mode == 4) return custom_amplitude(p, dx, dy);
    const float radius = sqrtf(dx * dx + dy * dy);
    bool inside;
    switch (p.mode) {
        case 0: inside = radius <= kOuterRadius; break;
        case 2: inside = star_metric(dx, dy, p.sides, p.star_inner, p.rotation) <= 1.0f; break;
        case 3: inside = spiral_open(p, dx, dy); break;
        case 6: inside = square_grid_open(p, dx, dy); break;
        case 7: inside = snowflake_open(p, dx, dy); break;
        default: inside = polygon_metric(dx, dy, p.sides, p.roundness, p.rotation) <= 1.0f; break;
    }
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
    if (radius <= start) return 1.0f;  // t = 0 below: cos(0) = 1 exactly
    const float t = fminf(fmaxf((radius - start) / fmaxf(fade, 1e-6f), 0.0f), 1.0f);
    const float s = t * t * (3.0f - 2.0f * t);
    return fmaxf(0.0f, cosf(s * static_cast<float>(3.14159265358979323846 * 0.5)));
}

}  // namespace ld
