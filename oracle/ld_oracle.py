"""FP64 CPU restatement of the LensDiff diffraction path — TEST INFRASTRUCTURE.

This module is the checker for the CUDA path: only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg may import it.  The
product (lensdiff_b200) never calls it and has no CPU fallback.

Pinning: every stage here is checked against the reference's own CPU code,
compiled from its sources into oracle/_ref/libldref.so (oracle/Makefile,
oracle/ref_shim.cpp), by tests/test_oracle_vs_reference.py, and against the
golden fixtures in tests/golden/ that tests/golden/make_golden.py generated
from that library.  Configurations the reference cannot express (more than 9
wavelengths, Gaussian RGB responses, Noll terms outside 4..17, field grids
other than 3x3) are pinned only through reduction cases that coincide with a
reference configuration.

Arithmetic: discrete decisions (pupil inside/outside tests, sample positions,
radius rounding) follow the reference's float32 expressions; transforms,
sums and values are float64.  Every function names the reference lines it
restates (paths relative to the reference project root).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

try:  # the same FP64 transforms, spread over the host's cores
    import os as _os

    import scipy.fft as _sfft

    _WORKERS = max(1, _os.cpu_count() or 1)

    def _fft2(x):
        return _sfft.fft2(x, workers=_WORKERS)

    def _rfft2(x, s=None):
        return _sfft.rfft2(x, s, workers=_WORKERS)

    def _irfft2(x, s):
        return _sfft.irfft2(x, s, workers=_WORKERS)
except ImportError:  # numpy's pocketfft, one core
    def _fft2(x):
        return np.fft.fft2(x)

    def _rfft2(x, s=None):
        return np.fft.rfft2(x, s)

    def _irfft2(x, s):
        return np.fft.irfft2(x, s)

F = np.float32
K_PI_F = F(3.14159265358979323846)  # kPi, LensDiffCpuReference.cpp:25
GRAY18 = F(0.18)
OUTER_RADIUS = F(0.86)  # LensDiffCpuReference.cpp:766


def _p(params, name, default=None):
    return getattr(params, name, default)


# --------------------------------------------------------------------------
# Sizes (LensDiffTypes.h:292-320, LensDiffCpuReference.cpp:104-115)
# --------------------------------------------------------------------------
def optics_short_side(p) -> int:
    """ResolveLensDiffOpticsShortSidePx, LensDiffTypes.h:302-305."""
    if _p(p, "resolutionAware", False):
        return 2160
    return max(1, int(p.frameShortSidePx))


def percent_to_px(percent: float, short_side: int) -> float:
    """ResolveLensDiffAuthoringPercentToPixels, LensDiffTypes.h:312-314 (double)."""
    return max(0.0, float(percent)) * 0.01 * float(max(1, short_side))


def max_kernel_radius(p) -> int:
    """max(4, ResolveLensDiffMaxKernelRadiusPx), LensDiffTypes.h:316-320 / CpuReference.cpp:1710."""
    r = max(0, int(math.ceil(percent_to_px(p.maxKernelRadiusPx, optics_short_side(p)))))
    return max(4, r)


def pupil_size(p) -> int:
    """effectivePupilResolution, LensDiffCpuReference.cpp:104-106."""
    return min(max(int(p.pupilResolution), 64), 1024)


def raw_psf_size(np_: int, rmax: int) -> int:
    """chooseRawPsfSize, LensDiffCpuReference.cpp:112-115."""
    return min(max(max(np_ * 2, max(512, rmax * 4)), 128), 16384)


def resolve_sizes(p) -> Tuple[int, int, int]:
    np_ = pupil_size(p)
    rmax = max_kernel_radius(p)
    return np_, raw_psf_size(np_, rmax), rmax


MODE_WAVELENGTHS = {
    0: [550.0],
    1: [460.0, 550.0, 610.0],
    2: [440.0, 490.0, 540.0, 590.0, 640.0],
    3: [420.0, 450.0, 480.0, 510.0, 540.0, 570.0, 600.0, 630.0, 660.0],
}


def wavelengths(p) -> List[float]:
    """wavelengthsForMode (LensDiffCpuReference.cpp:1602-1614) or the explicit list."""
    w = _p(p, "wavelengthsNm", None)
    if w:
        return [float(F(x)) for x in w]
    return MODE_WAVELENGTHS[int(p.spectralMode)]


# --------------------------------------------------------------------------
# Pupil amplitude (LensDiffCpuReference.cpp:451-488, :670-680, :758-822)
# --------------------------------------------------------------------------
def _pixel_coords(size: int):
    x = ((np.arange(size, dtype=F) + F(0.5)) / F(size) - F(0.5)) * F(2.0)
    nx, ny = np.meshgrid(x, x)  # ny varies along rows
    return nx.astype(F), ny.astype(F)


def _rotation_rad(p) -> np.float32:
    return F(float(p.rotationDeg) * float(K_PI_F) / 180.0)


def polygon_metric(nx, ny, blade_count: int, roundness: np.float32, rotation: np.float32,
                   outer: np.float32):
    """polygonMetric, LensDiffCpuReference.cpp:451-469 (float32 expressions)."""
    radius = np.sqrt(nx * nx + ny * ny).astype(F)
    circle = (radius / max(outer, F(1e-5))).astype(F)
    if blade_count < 3:
        return circle
    angle = (np.arctan2(ny, nx).astype(F) - rotation).astype(F)
    sector = F(F(2.0) * K_PI_F / F(blade_count))
    local = np.fmod(angle, sector).astype(F)
    local = np.where(local < 0, (local + sector).astype(F), local).astype(F)
    local = (local - sector * F(0.5)).astype(F)
    poly_r = (outer * F(np.cos(K_PI_F / F(blade_count))) /
              np.maximum(np.cos(local).astype(F), F(1e-4))).astype(F)
    poly_metric = (radius / np.maximum(poly_r, F(1e-5))).astype(F)
    return (circle * roundness + poly_metric * (F(1.0) - roundness)).astype(F)


def blocked_by_vanes(nx, ny, vane_count: int, thickness: np.float32, rotation: np.float32,
                     outer: np.float32):
    """blockedByVanes, LensDiffCpuReference.cpp:471-488."""
    blocked = np.zeros(nx.shape, dtype=bool)
    if vane_count <= 0 or thickness <= 0:
        return blocked
    scaled = F(thickness * outer)
    n = max(1, vane_count)
    for i in range(n):
        ang = F(rotation + F(i) * K_PI_F / F(n))
        cs, sn = F(np.cos(ang)), F(np.sin(ang))
        xr = (nx * cs + ny * sn).astype(F)
        yr = (-nx * sn + ny * cs).astype(F)
        blocked |= (np.abs(yr) <= scaled) & (np.abs(xr) <= outer)
    return blocked


def apodization(mode: int, radial_norm):
    """apodizationWeight, LensDiffCpuReference.cpp:670-680."""
    if mode == 1:
        return np.cos(np.minimum(radial_norm, F(1.0)) * (K_PI_F * F(0.5))).astype(F)
    if mode == 2:
        return np.exp(F(-4.0) * radial_norm * radial_norm).astype(F)
    return np.ones_like(radial_norm, dtype=F)


def prepared_aperture_image(values: np.ndarray, normalize: bool, invert: bool) -> np.ndarray:
    """LoadLensDiffPreparedApertureImage, LensDiffApertureImage.cpp:367-399, on
    an already decoded amplitude image (float32)."""
    v = np.asarray(values, dtype=F).copy()
    lo, hi = F(v.min()), F(v.max())
    if normalize and hi > lo:
        scale = F(F(1.0) / F(hi - lo))
        v = np.clip(((v - lo).astype(F) * scale).astype(F), F(0.0), F(1.0)).astype(F)
    if invert:
        v = (F(1.0) - v).astype(F)
    return v


def custom_pupil_amplitude(p, image: np.ndarray) -> np.ndarray:
    """buildCustomPupilAmplitude, LensDiffCpuReference.cpp:707-756, with the
    bilinear sampleImageBilinear of :682-705 (float32 expressions)."""
    size = pupil_size(p)
    h, w = image.shape
    nx, ny = _pixel_coords(size)
    dx = (nx - F(p.pupilDecenterX)).astype(F)
    dy = (ny - F(p.pupilDecenterY)).astype(F)
    radius = np.sqrt((dx * dx + dy * dy).astype(F)).astype(F)
    rot = _rotation_rad(p)
    cs, sn = F(np.cos(-rot)), F(np.sin(-rot))
    aspect = F(F(w) / F(max(1, h)))
    fw = F(1.0) if aspect >= F(1.0) else aspect
    fh = F(F(1.0) / aspect) if aspect >= F(1.0) else F(1.0)
    rx = (dx * cs - dy * sn).astype(F)
    ry = (dx * sn + dy * cs).astype(F)
    ux = (rx / OUTER_RADIUS).astype(F)
    uy = (ry / OUTER_RADIUS).astype(F)
    keep = (radius <= OUTER_RADIUS) & (np.abs(ux) <= fw) & (np.abs(uy) <= fh)
    sx = (((ux / fw).astype(F) * F(0.5) + F(0.5)).astype(F) * F(w - 1)).astype(F)
    sy = (((uy / fh).astype(F) * F(0.5) + F(0.5)).astype(F) * F(h - 1)).astype(F)
    inside = (sx >= 0) & (sy >= 0) & (sx <= F(w - 1)) & (sy <= F(h - 1))
    xs = np.where(inside, sx, F(0)).astype(F)
    ys = np.where(inside, sy, F(0)).astype(F)
    x0 = np.floor(xs).astype(np.int64)
    y0 = np.floor(ys).astype(np.int64)
    x1 = np.minimum(x0 + 1, w - 1)
    y1 = np.minimum(y0 + 1, h - 1)
    tx = (xs - x0.astype(F)).astype(F)
    ty = (ys - y0.astype(F)).astype(F)
    img = image.astype(F)
    vx0 = (img[y0, x0] + (img[y0, x1] - img[y0, x0]) * tx).astype(F)
    vx1 = (img[y1, x0] + (img[y1, x1] - img[y1, x0]) * tx).astype(F)
    sample = np.where(inside, (vx0 + (vx1 - vx0) * ty).astype(F), F(0))
    amp = (sample * apodization(int(p.apodizationMode), (radius / OUTER_RADIUS).astype(F))).astype(F)
    return np.where(keep, amp, F(0)).astype(F)


def pupil_amplitude(p) -> np.ndarray:
    """buildPupilAmplitude, LensDiffCpuReference.cpp:758-822 (Circle/Polygon/Hexagon;
    Custom through custom_pupil_amplitude with the decoded image of
    p.customApertureImage)."""
    size = pupil_size(p)
    mode = int(p.apertureMode)
    if mode == 4:
        img = getattr(p, "customApertureImage", None)
        if img is None:
            raise ValueError("Custom aperture without a decoded image")
        prepared = prepared_aperture_image(img, bool(p.customApertureNormalize), bool(p.customApertureInvert))
        return custom_pupil_amplitude(p, prepared)
    if mode not in (0, 1, 5):
        raise NotImplementedError(f"aperture mode {mode} is not restated")
    nx, ny = _pixel_coords(size)
    dx = (nx - F(p.pupilDecenterX)).astype(F)
    dy = (ny - F(p.pupilDecenterY)).astype(F)
    radius = np.sqrt(dx * dx + dy * dy).astype(F)
    outer = OUTER_RADIUS
    obstruction = F(F(max(0.0, min(0.95, float(p.centralObstruction)))) * outer)
    rotation = _rotation_rad(p)
    roundness = F(min(max(float(p.roundness), 0.0), 1.0))
    thickness = F(max(0.0, float(p.vaneThickness)))
    if mode == 0:
        inside = radius <= outer
    else:
        sides = 6 if mode == 5 else max(3, int(p.bladeCount))
        inside = polygon_metric(dx, dy, sides, roundness, rotation, outer) <= F(1.0)
    keep = inside & ~(radius < obstruction)
    keep &= ~blocked_by_vanes(dx, dy, int(p.vaneCount), thickness, rotation, outer)
    amp = apodization(int(p.apodizationMode), (radius / outer).astype(F))
    return np.where(keep, amp, F(0)).astype(F)


# --------------------------------------------------------------------------
# Zernike phase (LensDiffPhase.cpp:9-16, :20-38, :170-243)
# --------------------------------------------------------------------------
NAMED_TERMS = [  # (params field, Noll index) — LensDiffPhase.cpp:182-197
    ("phaseDefocus", 4), ("phaseAstigmatism45", 5), ("phaseAstigmatism0", 6),
    ("phaseComaY", 7), ("phaseComaX", 8), ("phaseTrefoilY", 9), ("phaseTrefoilX", 10),
    ("phaseSpherical", 11), ("phaseSecondaryAstigmatism0", 12),
    ("phaseSecondaryAstigmatism45", 13), ("phaseQuadrafoil0", 14), ("phaseQuadrafoil45", 15),
    ("phaseSecondaryComaX", 16), ("phaseSecondaryComaY", 17),
]


def noll_coefficients(p, defocus_override: Optional[float] = None) -> np.ndarray:
    """Named terms (LensDiffPhase.cpp:199-212) plus the extension Noll vector."""
    c = np.zeros(23, dtype=np.float64)
    for name, j in NAMED_TERMS:
        c[j] += float(getattr(p, name))
    if defocus_override is not None:
        c[4] = defocus_override + (c[4] - float(p.phaseDefocus))
    extra = _p(p, "noll", None)
    if extra is not None:
        for j, v in enumerate(list(extra)[:23]):
            c[j] += float(v)
    return c


def has_nonflat_phase(p, coeffs: np.ndarray, phase_enabled: bool) -> bool:
    """HasLensDiffNonFlatPhase, LensDiffPhase.cpp:20-38 (plus extension terms)."""
    if not phase_enabled:
        return False
    if np.any(np.abs(coeffs[1:]) > 1e-6):
        return True
    return abs(float(p.pupilDecenterX)) > 1e-6 or abs(float(p.pupilDecenterY)) > 1e-6


def zernike_terms(sx, sy):
    """Noll-indexed normalised Zernike terms.  j = 4..17 restate
    LensDiffPhase.cpp:182-197 in float32; j = 1..3 and 18..22 are the standard
    Noll definitions (extension, not in the reference)."""
    r2 = (sx * sx + sy * sy).astype(F)
    t = {}
    t[1] = np.ones_like(sx, dtype=F)
    t[2] = (F(2.0) * sx).astype(F)
    t[3] = (F(2.0) * sy).astype(F)
    t[4] = (F(1.7320508075688772) * (F(2.0) * r2 - F(1.0))).astype(F)
    t[6] = (F(2.4494897427831781) * (sx * sx - sy * sy)).astype(F)
    t[5] = (F(2.4494897427831781) * (F(2.0) * sx * sy)).astype(F)
    t[8] = (F(2.8284271247461901) * ((F(3.0) * r2 - F(2.0)) * sx)).astype(F)
    t[7] = (F(2.8284271247461901) * ((F(3.0) * r2 - F(2.0)) * sy)).astype(F)
    t[11] = (F(2.2360679774997898) * (F(6.0) * r2 * r2 - F(6.0) * r2 + F(1.0))).astype(F)
    t[10] = (F(2.8284271247461901) * (sx * sx * sx - F(3.0) * sx * sy * sy)).astype(F)
    t[9] = (F(2.8284271247461901) * (F(3.0) * sx * sx * sy - sy * sy * sy)).astype(F)
    sar = (F(4.0) * r2 - F(3.0)).astype(F)
    t[12] = (F(3.1622776601683795) * sar * (sx * sx - sy * sy)).astype(F)
    t[13] = (F(3.1622776601683795) * sar * (F(2.0) * sx * sy)).astype(F)
    t[14] = (F(3.1622776601683795) * (sx * sx * sx * sx - F(6.0) * sx * sx * sy * sy + sy * sy * sy * sy)).astype(F)
    t[15] = (F(3.1622776601683795) * (F(4.0) * sx * sy * (sx * sx - sy * sy))).astype(F)
    scr = (F(10.0) * r2 * r2 - F(12.0) * r2 + F(3.0)).astype(F)
    t[16] = (F(3.4641016151377544) * scr * sx).astype(F)
    t[17] = (F(3.4641016151377544) * scr * sy).astype(F)
    # extension terms (standard Noll, even j -> cos m*theta, odd j -> sin m*theta)
    x2, y2 = sx * sx, sy * sy
    cos3 = sx * (x2 - F(3.0) * y2)           # r^3 cos 3t
    sin3 = sy * (F(3.0) * x2 - y2)           # r^3 sin 3t
    r3rad = (F(5.0) * r2 - F(4.0)).astype(F)  # (5 r^5 - 4 r^3) / r^3
    t[18] = (F(3.4641016151377544) * r3rad * cos3).astype(F)
    t[19] = (F(3.4641016151377544) * r3rad * sin3).astype(F)
    c5 = sx * (x2 * x2 - F(10.0) * x2 * y2 + F(5.0) * y2 * y2)  # r^5 cos 5t
    s5 = sy * (F(5.0) * x2 * x2 - F(10.0) * x2 * y2 + y2 * y2)  # r^5 sin 5t
    t[20] = (F(3.4641016151377544) * c5).astype(F)
    t[21] = (F(3.4641016151377544) * s5).astype(F)
    t[22] = (F(2.6457513110645906) * (F(20.0) * r2 * r2 * r2 - F(30.0) * r2 * r2 + F(12.0) * r2 - F(1.0))).astype(F)
    return t


def phase_waves(p, coeffs: np.ndarray, phase_enabled: bool) -> np.ndarray:
    """BuildLensDiffPupilPhaseWaves, LensDiffPhase.cpp:215-243 with
    EvaluateLensDiffPhaseWaves :170-213."""
    size = pupil_size(p)
    out = np.zeros((size, size), dtype=F)
    if not has_nonflat_phase(p, coeffs, phase_enabled):
        return out
    rot = _rotation_rad(p)
    cs, sn = F(np.cos(-rot)), F(np.sin(-rot))
    nx, ny = _pixel_coords(size)
    radius = np.sqrt(nx * nx + ny * ny).astype(F)
    rx = (nx * cs - ny * sn).astype(F)
    ry = (nx * sn + ny * cs).astype(F)
    px = (rx / OUTER_RADIUS).astype(F)
    py = (ry / OUTER_RADIUS).astype(F)
    sx = (px - F(p.pupilDecenterX)).astype(F)
    sy = (py - F(p.pupilDecenterY)).astype(F)
    r2 = (sx * sx + sy * sy).astype(F)
    terms = zernike_terms(sx, sy)
    val = np.zeros((size, size), dtype=np.float64)
    for j in range(1, 23):
        if coeffs[j] != 0.0:
            val += float(F(coeffs[j])) * terms[j].astype(np.float64)
    val = val.astype(F)
    valid = (radius <= OUTER_RADIUS) & (r2 <= F(1.0))
    out[valid] = val[valid]
    return out


def wavelength_phase_setup(p, wavelength: float):
    """Per-wavelength defocus offset and phase enable, LensDiffCpuReference.cpp:1721-1727."""
    offset = F((F(wavelength) - F(550.0)) / F(110.0))
    defocus = float(p.phaseDefocus) + float(p.chromaticFocus) * float(offset)
    enabled = int(p.phaseMode) == 1 or abs(defocus) > 1e-6
    coeffs = noll_coefficients(p, defocus_override=defocus)
    return coeffs, enabled, offset


# --------------------------------------------------------------------------
# Raw PSF (LensDiffCpuReference.cpp:831-859, :303-314, :440-449)
# --------------------------------------------------------------------------
def fft_shift_square(img: np.ndarray) -> np.ndarray:
    """fftShiftSquare, LensDiffCpuReference.cpp:303-314: out[y,x] = in[(y+S/2)%S, (x+S/2)%S]."""
    half = img.shape[0] // 2
    return np.roll(img, (-half, -half), axis=(0, 1))


def raw_psf(amplitude: np.ndarray, phase: Optional[np.ndarray], size: int,
            normalize: bool = True) -> np.ndarray:
    """buildShiftedRawPsf: embed A*exp(i 2pi phi) at (S-N)/2, 2D DFT, |.|^2,
    fftshift, normalise (LensDiffCpuReference.cpp:831-859)."""
    n = amplitude.shape[0]
    off = max(0, (size - n) // 2)
    a = amplitude.astype(np.float64)
    field = a.astype(np.complex128)
    if phase is not None and phase.shape == amplitude.shape:
        ang = np.where(a > 0, phase.astype(np.float64) * 2.0 * math.pi, 0.0)
        field = a * np.exp(1j * ang)
    grid = np.zeros((size, size), dtype=np.complex128)
    grid[off:off + n, off:off + n] = field[: size - off, : size - off]
    spec = _fft2(grid)
    inten = spec.real ** 2 + spec.imag ** 2
    inten = fft_shift_square(inten)
    if normalize:
        tot = inten.sum()
        if tot > 0:
            inten = inten / tot
    return inten


def spectrum_center(size: int) -> np.float32:
    """shiftedSpectrumCenterCoordinate, LensDiffCpuReference.cpp:108-110."""
    return F(size * 0.5) if size % 2 == 0 else F((size - 1) * 0.5)


def first_minimum_radius(psf: np.ndarray) -> float:
    """estimateFirstMinimumRadius with radialMeanProfile and refineParabolicMinimum,
    LensDiffCpuReference.cpp:865-955."""
    size = psf.shape[0]
    rmax = size // 2
    c = spectrum_center(size)
    idx = (np.arange(size, dtype=F) - c).astype(F)
    dx, dy = np.meshgrid(idx, idx)
    rr = np.sqrt(dx * dx + dy * dy).astype(F).astype(np.float64)
    ri = np.minimum(rmax, np.floor(rr + 0.5).astype(np.int64))  # std::round, r >= 0
    sums = np.bincount(ri.ravel(), psf.ravel().astype(np.float64), minlength=rmax + 1)
    cnt = np.bincount(ri.ravel(), minlength=rmax + 1)
    prof = sums / np.maximum(cnt, 1)
    if prof.size < 4:
        return 1.0
    sm = np.empty_like(prof)
    n = prof.size
    for i in range(n):
        left = prof[0 if i == 0 else i - 1]
        right = prof[i + 1 if i + 1 < n else i]
        sm[i] = (left + 2.0 * prof[i] + right) * 0.25

    def refine(l, cc, r):
        den = l - 2.0 * cc + r
        if abs(den) < 1e-6:
            return 0.0
        return min(max(0.5 * (l - r) / den, -0.5), 0.5)

    best = 1
    bestv = sm[1]
    desc = 1 if sm[1] < sm[0] else 0
    for i in range(2, n - 1):
        if sm[i] <= sm[i - 1]:
            desc += 1
            if sm[i] < bestv:
                bestv = sm[i]
                best = i
            continue
        if desc >= 2 and best > 0 and best + 1 < n:
            return max(1.0, best + refine(sm[best - 1], sm[best], sm[best + 1]))
        best = i
        bestv = sm[i]
        desc = 0
    limit = max(2, min(n - 1, max(4, size // 8)))
    best = 1
    bestv = sm[1]
    for i in range(2, limit + 1):
        if sm[i] < bestv:
            bestv = sm[i]
            best = i
    if best > 0 and best + 1 < n:
        return max(1.0, best + refine(sm[best - 1], sm[best], sm[best + 1]))
    return float(best)


def reference_first_zero(np_: int, size: int) -> float:
    """GetLensDiffReferenceRawPsfCached + estimateFirstMinimumRadius for the clear
    circle, LensDiffCpuReference.cpp:2018-2038 and :1713-1714."""
    class _Circle:
        apertureMode = 0
        apodizationMode = 0
        pupilResolution = np_
        pupilDecenterX = 0.0
        pupilDecenterY = 0.0
        centralObstruction = 0.0
        rotationDeg = 0.0
        roundness = 1.0
        vaneThickness = 0.01
        vaneCount = 0
        bladeCount = 6
    amp = pupil_amplitude(_Circle)
    return first_minimum_radius(raw_psf(amp, None, size))


# --------------------------------------------------------------------------
# lambda-rescale (LensDiffCpuReference.cpp:316-353, :1060-1086)
# --------------------------------------------------------------------------
def _bilinear(img: np.ndarray, x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """sampleSquareBilinear, LensDiffCpuReference.cpp:316-336 (float32 coordinates)."""
    size = img.shape[0]
    lim = F(size - 1)
    bad = (x < 0) | (y < 0) | (x > lim) | (y > lim)
    xs = np.where(bad, F(0), x)
    ys = np.where(bad, F(0), y)
    x0 = np.floor(xs).astype(np.int64)
    y0 = np.floor(ys).astype(np.int64)
    x1 = np.minimum(x0 + 1, size - 1)
    y1 = np.minimum(y0 + 1, size - 1)
    tx = (xs - x0.astype(F)).astype(np.float64)
    ty = (ys - y0.astype(F)).astype(np.float64)
    v00 = img[y0, x0]
    v10 = img[y0, x1]
    v01 = img[y1, x0]
    v11 = img[y1, x1]
    vx0 = v00 + (v10 - v00) * tx
    vx1 = v01 + (v11 - v01) * tx
    return np.where(bad, 0.0, vx0 + (vx1 - vx0) * ty)


def resample_kernel(raw: np.ndarray, scale: float, radius: int) -> np.ndarray:
    """makeResampledKernel with sampleSquareFiltered, LensDiffCpuReference.cpp:338-353, :1060-1086."""
    size = raw.shape[0]
    ksize = 2 * radius + 1
    rc = spectrum_center(size)
    kc = F(F(ksize - 1) * F(0.5))
    inv = F(F(1.0) / max(F(scale), F(0.05)))
    d = (np.arange(ksize, dtype=F) - kc).astype(F)
    dx, dy = np.meshgrid(d, d)
    sx = (rc + dx * inv).astype(F)
    sy = (rc + dy * inv).astype(F)
    if inv <= F(1.0):
        k = _bilinear(raw, sx, sy)
    else:
        taps = min(max(int(math.ceil(float(inv))), 2), 6)
        step = F(inv / F(taps))
        acc = np.zeros((ksize, ksize), dtype=np.float64)
        for ty in range(taps):
            oy = F(F(F(ty) + F(0.5)) * step - inv * F(0.5))
            for tx in range(taps):
                ox = F(F(F(tx) + F(0.5)) * step - inv * F(0.5))
                acc += _bilinear(raw, (sx + ox).astype(F), (sy + oy).astype(F))
        k = acc / float(taps * taps)
    tot = k.sum()
    return k / tot if tot > 0 else k


def wavelength_scale(scale_base: np.float32, wavelength: float, chromatic_spread: float) -> np.float32:
    """scaleFactor, LensDiffCpuReference.cpp:1722, :1729-1730 (float32)."""
    w = F(wavelength)
    off = F((w - F(550.0)) / F(110.0))
    chrom = max(F(0.25), F(F(1.0) + F(chromatic_spread) * off))
    return F(F(scale_base * F(w / F(550.0))) * chrom)


def scale_base(p, r0: float) -> np.float32:
    """scaleBase, LensDiffCpuReference.cpp:1714-1715."""
    diff_px = percent_to_px(p.diffractionScalePx, optics_short_side(p))
    return F(F(max(1.0, diff_px)) / max(F(1.0), F(r0)))


# --------------------------------------------------------------------------
# Kernel shaping (LensDiffCpuReference.cpp:957-1151, :1616-1656)
# --------------------------------------------------------------------------
def _centered_radius(ksize: int) -> np.ndarray:
    c = F(F(ksize - 1) * F(0.5))
    d = (np.arange(ksize, dtype=F) - c).astype(F)
    dx, dy = np.meshgrid(d, d)
    return np.sqrt(dx * dx + dy * dy).astype(F)


def normalize(k: np.ndarray) -> np.ndarray:
    """normalizeKernel, LensDiffCpuReference.cpp:440-449."""
    t = k.sum()
    return k / t if t > 0 else k


def azimuthal_mean(k: np.ndarray) -> np.ndarray:
    """azimuthalMeanKernel, LensDiffCpuReference.cpp:1088-1120."""
    ksize = k.shape[0]
    rmax = ksize // 2
    ri = np.minimum(rmax, np.floor(_centered_radius(ksize).astype(np.float64) + 0.5).astype(np.int64))
    sums = np.bincount(ri.ravel(), k.ravel(), minlength=rmax + 1)
    cnt = np.bincount(ri.ravel(), minlength=rmax + 1)
    mean = (sums / np.maximum(cnt, 1))[ri]
    return normalize(mean)


def reshape_anisotropy(base: np.ndarray, mean: np.ndarray, emphasis: float) -> np.ndarray:
    """reshapeAnisotropy, LensDiffCpuReference.cpp:1122-1135."""
    gain = 1.0 + max(0.0, float(F(emphasis))) * 4.0
    return normalize(np.maximum(0.0, mean + (base - mean) * gain))


def positive_residual(full: np.ndarray, mean: np.ndarray) -> np.ndarray:
    """positiveResidualKernel, LensDiffCpuReference.cpp:1137-1151."""
    return normalize(np.maximum(0.0, full - mean))


def adaptive_support_radius(k: np.ndarray, max_radius: int) -> int:
    """estimateAdaptiveSupportRadius, LensDiffCpuReference.cpp:984-1031."""
    ksize = k.shape[0]
    rmax = min(max_radius, ksize // 2)
    ri = np.minimum(rmax, np.ceil(_centered_radius(ksize).astype(np.float64)).astype(np.int64))
    energy = np.bincount(ri.ravel(), k.ravel(), minlength=rmax + 1)
    peak = np.zeros(rmax + 1)
    np.maximum.at(peak, ri.ravel(), k.ravel())
    total = k.sum()
    gpeak = k.max()
    if total <= 1e-6 or gpeak <= 1e-6:
        return max(4, rmax)
    outside = np.zeros(rmax + 2)
    for r in range(rmax, -1, -1):
        outside[r] = max(peak[r], outside[r + 1])
    cum = np.cumsum(energy)
    for r in range(rmax + 1):
        captured = cum[r] / total
        remaining = outside[min(rmax + 1, r + 1)]
        if captured >= float(F(0.9999)) and remaining <= gpeak * float(F(2e-4)):
            return max(4, r + 1)
    return max(4, rmax)


def padded_support_radius(est: int, max_radius: int) -> int:
    """paddedAdaptiveSupportRadius, LensDiffCpuReference.cpp:1033-1036."""
    pad = max(6, min(24, int(math.ceil(float(F(F(max(1, est)) * F(0.05)))))))
    return min(max(est + pad, 4), max(4, max_radius))


def taper_weights(ksize: int, support: int) -> np.ndarray:
    """applySupportBoundaryTaper, LensDiffCpuReference.cpp:957-982."""
    extent = F(max(1.0, float(support)))
    fade = F(max(F(6.0), min(F(24.0), F(extent * F(0.04)))))
    start = F(max(F(0.0), F(extent - fade)))
    r = _centered_radius(ksize)
    t = np.clip(((r - start) / max(fade, F(1e-6))).astype(F), F(0.0), F(1.0)).astype(F)
    s = (t * t * (F(3.0) - F(2.0) * t)).astype(F)
    w = np.maximum(F(0.0), np.cos((s * F(math.pi * 0.5)).astype(F)).astype(F))
    return np.where(r >= extent, F(0.0), w).astype(np.float64)


def crop_kernel(k: np.ndarray, radius: int) -> np.ndarray:
    """cropKernelToRadius, LensDiffCpuReference.cpp:1038-1058."""
    ksize = k.shape[0]
    r = min(max(radius, 1), ksize // 2)
    c = ksize // 2
    out = k[c - r: c + r + 1, c - r: c + r + 1].copy()
    out = out * taper_weights(2 * r + 1, r)
    return normalize(out)


@dataclass
class PsfBin:
    wavelength: float
    full: np.ndarray
    core: np.ndarray
    structure: np.ndarray
    radius: int


def shape_bin(base: np.ndarray, wavelength: float, anisotropy: float, max_radius: int) -> PsfBin:
    """One bin of populatePsfBankCacheFromBaseKernels, LensDiffCpuReference.cpp:1633-1654."""
    mean = azimuthal_mean(base)
    shaped = reshape_anisotropy(base, mean, anisotropy)
    structure = positive_residual(shaped, mean)
    radius = padded_support_radius(adaptive_support_radius(shaped, max_radius), max_radius)
    return PsfBin(wavelength, crop_kernel(shaped, radius), crop_kernel(mean, radius),
                  crop_kernel(structure, radius), radius)


@dataclass
class PsfBank:
    bins: List[PsfBin]
    support_radius: int
    pupil: np.ndarray
    r0: float
    scale_base: float
    sizes: Tuple[int, int, int]


def build_psf_bank(p, r0: Optional[float] = None) -> PsfBank:
    """buildPsfBankGlobalOnly + populatePsfBankCacheFromBaseKernels,
    LensDiffCpuReference.cpp:1702-1734, :1616-1656."""
    np_, size, rmax = resolve_sizes(p)
    amp = pupil_amplitude(p)
    if r0 is None:
        r0 = reference_first_zero(np_, size)
    r0 = max(1.0, float(F(r0)))
    sb = scale_base(p, r0)
    bins = []
    support = 4
    for w in wavelengths(p):
        coeffs, enabled, _ = wavelength_phase_setup(p, w)
        ph = phase_waves(p, coeffs, enabled)
        raw = raw_psf(amp, ph, size)
        sc = wavelength_scale(sb, w, float(p.chromaticSpread))
        base = resample_kernel(raw, float(sc), rmax)
        b = shape_bin(base, w, float(p.anisotropyEmphasis), rmax)
        support = max(support, b.radius)
        bins.append(b)
    return PsfBank(bins, support, amp, r0, float(sb), (np_, size, rmax))


# --------------------------------------------------------------------------
# Spectral -> RGB (LensDiffSpectrum.cpp:362-376, :462-497)
# --------------------------------------------------------------------------
def gaussian_rgb_matrix(wl: Sequence[float], centers=(600.0, 540.0, 450.0), sigma=40.0) -> np.ndarray:
    """Extension: Gaussian RGB responses, each row normalised to unit sum."""
    w = np.asarray(wl, dtype=np.float64)
    m = np.stack([np.exp(-0.5 * ((w - float(F(c))) / float(F(sigma))) ** 2) for c in centers])
    return m / m.sum(axis=1, keepdims=True)


def map_bins(values: np.ndarray, natural: np.ndarray, style: np.ndarray, p) -> np.ndarray:
    """MapLensDiffSpectralBins, LensDiffSpectrum.cpp:462-497.  values: (..., B)."""
    b = values.shape[-1]
    if b <= 1:
        nat = np.repeat(values[..., :1], 3, axis=-1)
        sty = nat
    else:
        nat = values @ natural.T
        sty = values @ style.T
    force = min(max(float(F(p.spectrumForce)), 0.0), 1.0)
    rgb = np.maximum(0.0, nat * (1.0 - force) + sty * force)
    sat = max(0.0, float(p.spectrumSaturation))
    lw = np.array([0.2126, 0.7152, 0.0722])
    gray = rgb @ lw
    rgb = gray[..., None] + (rgb - gray[..., None]) * float(F(sat))
    if not bool(p.chromaticAffectsLuma):
        target = nat @ lw
        cur = rgb @ lw
        sc = np.where(cur > 1e-6, target / np.where(cur > 1e-6, cur, 1.0), 1.0)
        rgb = rgb * sc[..., None]
    return rgb


# --------------------------------------------------------------------------
# Highlight extraction (LensDiffCpuReference.cpp:1219-1279)
# --------------------------------------------------------------------------
def _luma(r, g, b):
    return F(0.2126) * r + F(0.7152) * g + F(0.0722) * b


def selection_mask(src: np.ndarray, p) -> np.ndarray:
    """buildSelectionMask, LensDiffCpuReference.cpp:1219-1249.  src: (H, W, 4) float32."""
    r, g, b = src[..., 0], src[..., 1], src[..., 2]
    soft = F(max(0.01, float(p.softnessStops)))
    thr = F(p.threshold)
    thr_lin = F(GRAY18 * F(np.power(F(2.0), thr)))
    maxrgb = np.maximum(np.maximum(r, g), b)
    signal = _luma(r, g, b).astype(F) if int(p.extractionMode) == 1 else maxrgb
    stops = np.log2(np.maximum(signal, F(1e-6)) / GRAY18).astype(np.float64)
    e0 = float(F(thr - soft * F(0.5)))
    e1 = float(F(thr + soft * F(0.5)))
    t = np.clip((stops - e0) / max(e1 - e0, 1e-4), 0.0, 1.0)
    gate = np.where(signal > 0, t * t * (3.0 - 2.0 * t), 0.0)
    boost = 1.0 + float(F(p.pointEmphasis)) * np.maximum(0.0, maxrgb.astype(np.float64) / max(float(thr_lin), 1e-4) - 1.0)
    return np.clip(gate * boost, 0.0, 1.0)


def extraction_signal(src: np.ndarray, p) -> np.ndarray:
    r, g, b = (src[..., i].astype(np.float64) for i in range(3))
    if int(p.extractionMode) == 1:
        return 0.2126 * r + 0.7152 * g + 0.0722 * b
    return np.maximum(np.maximum(r, g), b)


# --------------------------------------------------------------------------
# FFT convolution (LensDiffCpuReference.cpp:1153-1217)
# --------------------------------------------------------------------------
def convolve(plane: np.ndarray, kernel: np.ndarray) -> np.ndarray:
    """convolveScalar: zero-padded linear convolution with the kernel centred at
    (0,0), crop to the input, clamp >= 0 (LensDiffCpuReference.cpp:1167-1193).
    The grid is the exact linear size (W+K-1, H+K-1); linear convolution does
    not depend on the padding."""
    h, w = plane.shape
    k = kernel.shape[0]
    c = k // 2
    ph, pw = h + k - 1, w + k - 1
    kg = np.zeros((ph, pw))
    ys = (np.arange(k) - c) % ph
    xs = (np.arange(k) - c) % pw
    kg[np.ix_(ys, xs)] = kernel
    out = _irfft2(_rfft2(plane, (ph, pw)) * _rfft2(kg), (ph, pw))[:h, :w]
    return np.maximum(0.0, out)


def soft_shoulder(v: np.ndarray, shoulder: float) -> np.ndarray:
    """softShoulder, LensDiffCpuReference.cpp:81-87."""
    if shoulder <= 0:
        return np.maximum(0.0, v)
    x = np.maximum(0.0, v)
    return shoulder * (1.0 - np.exp(-x / shoulder))


# ---------------------------------------------------------------- field zones
FIELD_TERMS = [  # (radial, tangential, x target, y target, harmonic) — LensDiffPhase.cpp:131-166
    ("phaseFieldAstigRadial", "phaseFieldAstigTangential", "phaseAstigmatism0", "phaseAstigmatism45", 2),
    ("phaseFieldComaRadial", "phaseFieldComaTangential", "phaseComaX", "phaseComaY", 1),
    ("phaseFieldTrefoilRadial", "phaseFieldTrefoilTangential", "phaseTrefoilX", "phaseTrefoilY", 3),
    ("phaseFieldSecondaryAstigRadial", "phaseFieldSecondaryAstigTangential", "phaseSecondaryAstigmatism0",
     "phaseSecondaryAstigmatism45", 2),
    ("phaseFieldQuadrafoilRadial", "phaseFieldQuadrafoilTangential", "phaseQuadrafoil0", "phaseQuadrafoil45", 4),
    ("phaseFieldSecondaryComaRadial", "phaseFieldSecondaryComaTangential", "phaseSecondaryComaX",
     "phaseSecondaryComaY", 1),
]


def has_field_phase(p) -> bool:
    """HasLensDiffFieldPhase, LensDiffPhase.cpp:40-57."""
    if int(p.phaseMode) != 1 or abs(p.phaseFieldStrength) <= 1e-6:
        return False
    names = ["phaseFieldDefocus", "phaseFieldSpherical"] + [t[0] for t in FIELD_TERMS] + [t[1] for t in FIELD_TERMS]
    return any(abs(getattr(p, n)) > 1e-6 for n in names)


def resolve_field_zone(p, nx: float, ny: float):
    """ResolveLensDiffFieldZoneParams, LensDiffPhase.cpp:112-168 (FP64 as the
    reference): the zone's own Zernike coefficients; the field terms are
    cleared so the zone bank is built without zones."""
    q = p.copy()
    if not has_field_phase(p):
        return q
    radial = min(1.0, math.sqrt(float(nx) * nx + float(ny) * ny) / math.sqrt(2.0))
    bias = min(max(float(p.phaseFieldEdgeBias), 0.0), 1.0)
    scale = float(p.phaseFieldStrength) * radial ** (1.0 + bias * 2.0)
    q = q.copy(phaseFieldStrength=0.0)
    if abs(scale) <= 1e-9:
        return q
    ang = math.atan2(float(ny), float(nx))
    ch = {"phaseDefocus": p.phaseDefocus + p.phaseFieldDefocus * scale,
          "phaseSpherical": p.phaseSpherical + p.phaseFieldSpherical * scale}
    for rad, tan, xt, yt, h in FIELD_TERMS:
        rv, tv = getattr(p, rad) * scale, getattr(p, tan) * scale
        cs, sn = math.cos(h * ang), math.sin(h * ang)
        ch[xt] = getattr(p, xt) + rv * cs - tv * sn
        ch[yt] = getattr(p, yt) + rv * sn + tv * cs
    return q.copy(**ch)


def field_zone_weights(w: int, h: int, zx: int, zy: int, n: int = 3) -> np.ndarray:
    """accumulateWeightedImage tent weights, LensDiffCpuReference.cpp:1452-1475
    (float32 as the reference; n x n zones, the reference's n = 3)."""
    dx = F(max(1, w - 1))
    dy = F(max(1, h - 1))
    px = (np.arange(w, dtype=np.float32) / dx) * F(n - 1)
    py = (np.arange(h, dtype=np.float32) / dy) * F(n - 1)
    wx = np.maximum(F(0), F(1) - np.abs(px - F(zx)))
    wy = np.maximum(F(0), F(1) - np.abs(py - F(zy)))
    return (wy[:, None] * wx[None, :]).astype(np.float32)


def field_zone_banks(p, n: int = 3):
    """makeFieldZoneCache for every zone in the reference's order (zy outer,
    zx inner), LensDiffCpuReference.cpp:1779-1783."""
    out = []
    for zy in range(n):
        for zx in range(n):
            nx = 2.0 * zx / (n - 1) - 1.0
            ny = 2.0 * zy / (n - 1) - 1.0
            out.append((zx, zy, build_psf_bank(resolve_field_zone(p, F(nx), F(ny)))))
    return out


# ------------------------------------------------------------ transfer
def davinci_decode(x: np.ndarray) -> np.ndarray:
    """DaVinci Intermediate to linear (Blackmagic's published curve; the
    reference's decodeToLinear, ColorManagement.cpp:168-169), float."""
    x = np.asarray(x, np.float32)
    with np.errstate(over="ignore"):
        lin = (np.exp2(x / F(0.07329248) - F(7.0)) - F(0.0075)).astype(np.float32)
    return np.where(x <= F(0.02740668), (x / F(10.44426855)).astype(np.float32), lin)


def davinci_encode(x: np.ndarray) -> np.ndarray:
    """Linear to DaVinci Intermediate (encodeChannelFromLinear,
    LensDiffTransfer.cpp:8-20)."""
    x = np.asarray(x, np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        log = (np.log2(np.maximum(x, 0.0) + 0.0075) + 7.0) * 0.07329248
    return np.where(x <= 0.00262409, x * 10.44426855, log)


# ------------------------------------------------------- after the effect
def working_frame(p, w: int, h: int) -> Tuple[bool, int, int]:
    """Resolution-aware working frame: ResolveLensDiffEffectWorkingScale
    (LensDiffTypes.h:294-310) and the working size (CpuReference.cpp:2090-2093,
    std::lround of the double product)."""
    scale = float(optics_short_side(p)) / float(max(1, int(p.frameShortSidePx)))
    if not (_p(p, "resolutionAware", False) and abs(scale - 1.0) > 1e-6):
        return False, w, h
    return True, max(1, int(math.floor(w * scale + 0.5))), max(1, int(math.floor(h * scale + 0.5)))


def resample_rgba(img: np.ndarray, ow: int, oh: int) -> np.ndarray:
    """resampleRgbaImage (CpuReference.cpp:414-434) with
    sampleRgbaBilinearImage (:373-395): pixel centres mapped in float, zero
    outside [0, w-1] x [0, h-1], lerp form of the bilinear blend."""
    h, w = img.shape[:2]
    if (w, h) == (ow, oh):
        return img
    fx = ((np.arange(ow, dtype=np.float32) + F(0.5)) * (F(w) / F(max(1, ow))) - F(0.5)).astype(np.float32)
    fy = ((np.arange(oh, dtype=np.float32) + F(0.5)) * (F(h) / F(max(1, oh))) - F(0.5)).astype(np.float32)
    okx = (fx >= 0) & (fx <= F(w - 1))
    oky = (fy >= 0) & (fy <= F(h - 1))
    x0 = np.clip(np.floor(fx).astype(np.int64), 0, w - 1)
    y0 = np.clip(np.floor(fy).astype(np.int64), 0, h - 1)
    x1 = np.minimum(x0 + 1, w - 1)
    y1 = np.minimum(y0 + 1, h - 1)
    tx = (fx - x0.astype(np.float32)).astype(np.float64)[None, :, None]
    ty = (fy - y0.astype(np.float32)).astype(np.float64)[:, None, None]
    src = img.astype(np.float64)
    p00, p10 = src[np.ix_(y0, x0)], src[np.ix_(y0, x1)]
    p01, p11 = src[np.ix_(y1, x0)], src[np.ix_(y1, x1)]
    vx0 = p00 + (p10 - p00) * tx
    vx1 = p01 + (p11 - p01) * tx
    out = vx0 + (vx1 - vx0) * ty
    return out * (oky[:, None] & okx[None, :])[..., None]


def gaussian_kernel(radius_px: float) -> np.ndarray:
    """buildGaussianKernel, CpuReference.cpp:1680-1700: radius
    ceil(max(.5, r)), sigma max(.5, r / 2), values in float, normalised."""
    r = F(radius_px)
    rad = max(1, int(math.ceil(max(0.5, float(r)))))
    sigma = max(F(0.5), F(r * F(0.5)))
    yy, xx = np.mgrid[-rad:rad + 1, -rad:rad + 1]
    d = (xx * xx + yy * yy).astype(np.float32)
    v = np.exp(-(d / (F(2.0) * sigma * sigma))).astype(np.float32).astype(np.float64)
    return v / v.sum()


def _sample_clamped(plane: np.ndarray, fx: np.ndarray, fy: np.ndarray) -> np.ndarray:
    """sampleRgbaBilinear (CpuReference.cpp:1477-1497) on one channel:
    coordinates clamped to the frame, (1 - t) weights."""
    h, w = plane.shape
    x = np.clip(fx, F(0), F(max(0, w - 1))).astype(np.float32)
    y = np.clip(fy, F(0), F(max(0, h - 1))).astype(np.float32)
    x0 = np.floor(x).astype(np.int64)
    y0 = np.floor(y).astype(np.int64)
    x1 = np.minimum(x0 + 1, w - 1)
    y1 = np.minimum(y0 + 1, h - 1)
    tx = (x - x0.astype(np.float32)).astype(np.float64)
    ty = (y - y0.astype(np.float32)).astype(np.float64)
    a = plane[y0, x0] * (1.0 - tx) + plane[y0, x1] * tx
    b = plane[y1, x0] * (1.0 - tx) + plane[y1, x1] * tx
    return a * (1.0 - ty) + b * ty


def creative_fringe(effect: np.ndarray, amount: float) -> np.ndarray:
    """applyCreativeFringe, CpuReference.cpp:1499-1534: red sampled at +shift,
    blue at -shift along the direction from the frame centre (float
    geometry), green unshifted."""
    amt = F(amount)
    if amt <= F(1e-6):
        return effect
    h, w = effect.shape[:2]
    cx = F(max(0, w - 1)) * F(0.5)
    cy = F(max(0, h - 1)) * F(0.5)
    y, x = np.mgrid[0:h, 0:w]
    x = x.astype(np.float32)
    y = y.astype(np.float32)
    dx = (x - cx).astype(np.float32)
    dy = (y - cy).astype(np.float32)
    length = np.sqrt(dx * dx + dy * dy).astype(np.float32)
    with np.errstate(divide="ignore"):
        inv = np.where(length > F(1e-6), F(1.0) / length, F(0.0)).astype(np.float32)
    shx = (dx * inv * amt).astype(np.float32)
    shy = (dy * inv * amt).astype(np.float32)
    out = effect.copy()
    out[..., 0] = _sample_clamped(effect[..., 0], (x + shx).astype(np.float32), (y + shy).astype(np.float32))
    out[..., 2] = _sample_clamped(effect[..., 2], (x - shx).astype(np.float32), (y - shy).astype(np.float32))
    return out


def render(src: np.ndarray, p, bank: PsfBank, natural: Optional[np.ndarray] = None,
           style: Optional[np.ndarray] = None, src_origin=(0, 0), dst_bounds=None,
           render_window=None, field_grid: int = 3) -> np.ndarray:
    """RunLensDiffCpuReference, LensDiffCpuReference.cpp:2073-2261 (Final
    view).  With field phase on, `bank` is ignored and the effect is the
    tent-weighted sum of the zones' effects (:2161-2170); `field_grid` zones
    per side.  The effect is computed on the working frame (the source,
    resampled when resolution-aware, :2089-2094), then scattered, fringed
    and resampled back (:2180-2198) before the composite.

    src: (H, W, 4) float array at bounds origin `src_origin`.  Returns the dst
    image (dh, dw, 4) for `dst_bounds` = (x1, y1, x2, y2) (defaults to src)."""
    sh, sw = src.shape[:2]
    davinci = int(_p(p, "inputTransfer", 0)) == 1
    if davinci:  # loadSourceRgba decodes the source first (CpuReference.cpp:174-192)
        src = np.concatenate([davinci_decode(src[..., :3]), np.asarray(src[..., 3:4], np.float32)], axis=-1)
    srcd = src.astype(np.float64)
    resample, w, h = working_frame(p, sw, sh)
    work = resample_rgba(src, w, h).astype(np.float32) if resample else src
    mask = selection_mask(work, p)
    rscale = 1.0 - min(max(float(p.corePreserve), 0.0), 1.0)
    rscale = float(F(rscale))
    protect = max(0.2, float(F(min(max(float(p.corePreserve), 0.0), 1.0))))
    max_sub = (1.0 - protect) / rscale if rscale > 1e-6 else 0.0
    redist = work.astype(np.float64)[..., :3] * (mask * rscale)[..., None]
    driver = extraction_signal(work, p) * mask * rscale
    preserve = int(p.energyMode) == 0
    gain = min(max(float(p.effectGain), 0.0), 1.0) if preserve else max(0.0, float(p.effectGain))
    cc = gain if preserve else max(0.0, float(p.coreCompensation))
    spectral = int(p.spectralMode) != 0
    split = int(p.lookMode) == 1

    def effect_for(bk, kind: str) -> np.ndarray:
        if not spectral:
            ker = getattr(bk.bins[0], kind)
            return np.stack([convolve(redist[..., c], ker) for c in range(3)], axis=-1)
        planes = np.stack([convolve(driver, getattr(b, kind)) for b in bk.bins], axis=-1)
        return map_bins(planes, natural, style if style is not None else natural, p)

    def effect_of(bk) -> np.ndarray:
        if split:
            core = soft_shoulder(effect_for(bk, "core"), float(F(p.coreShoulder)))
            struct = soft_shoulder(effect_for(bk, "structure"), float(F(p.structureShoulder)))
            return core * max(0.0, float(p.coreGain)) + struct * max(0.0, float(p.structureGain))
        return effect_for(bk, "full")

    if has_field_phase(p):
        effect = np.zeros((h, w, 3))
        for zx, zy, bk in field_zone_banks(p, field_grid):
            effect += effect_of(bk) * field_zone_weights(w, h, zx, zy, field_grid)[..., None]
    else:
        effect = effect_of(bank)
    if preserve:
        lw = np.array([0.2126, 0.7152, 0.0722])
        e_in = float((redist @ lw).sum())
        e_fx = float((effect @ lw).sum())
        if e_fx > 1e-6:
            effect = effect * (e_in / e_fx)
    scatter_px = percent_to_px(_p(p, "scatterRadius", 0.0), optics_short_side(p))
    scatter_amount = float(_p(p, "scatterAmount", 0.0))
    if scatter_amount > 1e-6 and scatter_px > 0.25:
        g = gaussian_kernel(scatter_px)
        scat = np.stack([convolve(effect[..., c], g) for c in range(3)], axis=-1)
        effect = effect + scat * float(F(max(0.0, scatter_amount)))
    fringe_px = max(0.0, percent_to_px(_p(p, "creativeFringe", 0.0), optics_short_side(p)))
    effect = creative_fringe(effect, fringe_px)
    if resample:
        redist = resample_rgba(redist, sw, sh)
        effect = resample_rgba(effect, sw, sh)
    raw = np.maximum(0.0, srcd[..., :3] - cc * redist + gain * effect)
    floor = np.maximum(0.0, srcd[..., :3] - redist * max_sub)
    rgb = np.maximum(raw, floor)
    if davinci:  # the final pixels are encoded back (:2248-2250)
        rgb = davinci_encode(rgb)
    final = np.concatenate([rgb, srcd[..., 3:4]], axis=-1)
    h, w = sh, sw

    sx1, sy1 = src_origin
    if dst_bounds is None:
        dst_bounds = (sx1, sy1, sx1 + w, sy1 + h)
    if render_window is None:
        render_window = dst_bounds
    dx1, dy1, dx2, dy2 = dst_bounds
    out = np.zeros((dy2 - dy1, dx2 - dx1, 4))
    rx1, ry1 = max(render_window[0], dx1), max(render_window[1], dy1)
    rx2, ry2 = min(render_window[2], dx2), min(render_window[3], dy2)
    for y in range(ry1, max(ry1, ry2)):
        sy = y - sy1
        for x0 in [rx1]:
            xs = np.arange(rx1, max(rx1, rx2))
            sxv = xs - sx1
            ok = (sxv >= 0) & (sxv < w) & (0 <= sy < h)
            row = np.zeros((xs.size, 4))
            row[:, 3] = 1.0
            if 0 <= sy < h:
                row[ok] = final[sy, sxv[ok]]
            out[y - dy1, xs - dx1] = row
    return out
