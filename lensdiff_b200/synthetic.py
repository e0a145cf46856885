"""Seeded synthetic frames and lens settings for the benchmark workloads.

The reference publishes no benchmark data; these generators stand in for it
with the shapes, sizes and value distributions of the workloads the path is
measured on (a black frame with a 0-0.2 horizontal gradient, point
highlights at uniform-random pixels with log-uniform grey values, optional
anti-aliased line segments).
"""
from __future__ import annotations

import math
from typing import List, Optional

import numpy as np

from .types import (
    LensDiffApertureMode,
    LensDiffEnergyMode,
    LensDiffFftForm,
    LensDiffLookMode,
    LensDiffParams,
    LensDiffPhaseMode,
    LensDiffRgbMode,
    LensDiffSpectralMode,
)


def make_frame(width: int, height: int, points: int, lo: float, hi: float, seed: int,
               segments: int = 0, seg_lo: float = 5.0, seg_hi: float = 50.0) -> np.ndarray:
    """(H, W, 4) float32 RGBA: gradient 0 -> 0.2 in x, `points` log-uniform
    [lo, hi] grey highlights, `segments` 1-px anti-aliased line segments."""
    rng = np.random.default_rng(seed)
    img = np.zeros((height, width, 4), np.float32)
    grad = np.linspace(0.0, 0.2, width, dtype=np.float32)
    img[..., 0] = grad[None, :]
    img[..., 1] = grad[None, :]
    img[..., 2] = grad[None, :]
    img[..., 3] = 1.0
    xs = rng.integers(0, width, points)
    ys = rng.integers(0, height, points)
    vals = np.exp(rng.uniform(math.log(lo), math.log(hi), points)).astype(np.float32)
    for c in range(3):
        img[ys, xs, c] = vals
    for _ in range(segments):
        x0, x1 = rng.uniform(0, width - 1, 2)
        y0, y1 = rng.uniform(0, height - 1, 2)
        v = np.float32(rng.uniform(seg_lo, seg_hi))
        n = int(max(abs(x1 - x0), abs(y1 - y0))) + 1
        t = np.linspace(0.0, 1.0, n)
        px = x0 + (x1 - x0) * t
        py = y0 + (y1 - y0) * t
        # 1-px anti-aliased: split each sample bilinearly over its 4 neighbours
        ix = np.floor(px).astype(int)
        iy = np.floor(py).astype(int)
        fx = px - ix
        fy = py - iy
        for dx, dy, wgt in ((0, 0, (1 - fx) * (1 - fy)), (1, 0, fx * (1 - fy)),
                            (0, 1, (1 - fx) * fy), (1, 1, fx * fy)):
            xx = np.clip(ix + dx, 0, width - 1)
            yy = np.clip(iy + dy, 0, height - 1)
            for c in range(3):
                np.maximum.at(img[..., c], (yy, xx), (v * wgt).astype(np.float32))
    return img


def radius_percent(radius_px: int, short_side: int) -> float:
    """Percent value whose pixel radius ceil(percent * 0.01 * short_side) is
    exactly `radius_px` (the reference resolves percent to pixels in double
    precision and takes the ceiling, LensDiffTypes.h:312-320)."""
    pct = radius_px * 100.0 / short_side
    while math.ceil(max(0.0, pct) * 0.01 * float(short_side)) > radius_px:
        pct = math.nextafter(pct, 0.0)
    return pct


def base_params(short_side: int) -> LensDiffParams:
    """Settings shared by the workloads: Physical look, additive (Augment)
    blend with effect gain 1 and no core compensation, highlight threshold
    1.0 linear (log2(1/0.18) stops) with a 0.5-stop knee."""
    return LensDiffParams(
        lookMode=LensDiffLookMode.Physical,
        energyMode=LensDiffEnergyMode.Augment,
        effectGain=1.0,
        coreCompensation=0.0,
        corePreserve=0.0,
        threshold=math.log2(1.0 / 0.18),
        softnessStops=0.5,
        frameShortSidePx=short_side,
        diffractionScalePx=1.0,
        phaseMode=LensDiffPhaseMode.Enabled,
    )


def workload_small(seed: int = 1001):
    """1024x576, 64 highlights in [1,100], 6-blade polygon, pupil 256 -> PSF 512,
    defocus 0.25 + spherical 0.1 waves, 3 wavelengths 610/550/465 nm."""
    p = base_params(576)
    p.apertureMode = LensDiffApertureMode.Polygon
    p.bladeCount = 6
    p.roundness = 0.0
    p.pupilResolution = 256
    p.maxKernelRadiusPx = radius_percent(128, 576)
    p.phaseDefocus = 0.25
    p.phaseSpherical = 0.1
    p.spectralMode = LensDiffSpectralMode.Tristimulus
    p.wavelengthsNm = [610.0, 550.0, 465.0]
    p.rgbMode = LensDiffRgbMode.Gaussian
    frame = make_frame(1024, 576, 64, 1.0, 100.0, seed)
    return p, frame


def workload_hd(seed: int = 1002):
    """1920x1080, 512 highlights + 16 segments, 9 blades rounding 0.4,
    obstruction 0.3, 4 vanes of 0.02, pupil 512 -> 1024, Noll 2..15 ~ N(0, 0.1),
    16 wavelengths 400-700 nm with Gaussian RGB responses."""
    rng = np.random.default_rng(seed)
    p = base_params(1080)
    p.apertureMode = LensDiffApertureMode.Polygon
    p.bladeCount = 9
    p.roundness = 0.4
    p.centralObstruction = 0.3
    p.vaneCount = 4
    p.vaneThickness = 0.02 / 0.86  # 0.02 of the pupil diameter, in outer-radius units
    p.pupilResolution = 512
    p.maxKernelRadiusPx = radius_percent(256, 1080)
    noll = [0.0] * 23
    for j in range(2, 16):
        noll[j] = float(rng.normal(0.0, 0.1))
    p.noll = noll
    p.spectralMode = LensDiffSpectralMode.Spectral9
    p.wavelengthsNm = list(np.linspace(400.0, 700.0, 16))
    p.rgbMode = LensDiffRgbMode.Gaussian
    frame = make_frame(1920, 1080, 512, 1.0, 100.0, seed, segments=16)
    return p, frame


def workload_uhd31(seed: int = 1003, chromatic_focus: float = 0.2):
    """3840x2160, 2048 highlights in [1,1000], 31 wavelengths 400-700 nm at 10 nm,
    pupil 512 -> PSF 2048 (kernel radius up to 512 px), chromatic focus
    0.2 waves so every wavelength has its own pupil phase."""
    p = base_params(2160)
    p.apertureMode = LensDiffApertureMode.Polygon
    p.bladeCount = 6
    p.roundness = 0.0
    p.pupilResolution = 512
    p.maxKernelRadiusPx = radius_percent(512, 2160)
    p.phaseDefocus = 0.25
    p.phaseSpherical = 0.1
    p.chromaticFocus = chromatic_focus
    p.spectralMode = LensDiffSpectralMode.Spectral9
    p.wavelengthsNm = [400.0 + 10.0 * i for i in range(31)]
    p.rgbMode = LensDiffRgbMode.Gaussian
    frame = make_frame(3840, 2160, 2048, 1.0, 1000.0, seed)
    return p, frame


def workload_reference_uhd(seed: int = 1003):
    """The UHD frame and lens of workload_uhd31 at a setting the reference's
    own CUDA chain can express: its Spectral9 mode (9 wavelengths, its own
    spectral matrices), no chromatic focus, pupil 512 -> PSF 2048, kernel
    radius up to 512 px.  The same-GPU comparison with that chain runs here."""
    p, frame = workload_uhd31(seed, chromatic_focus=0.0)
    p.spectralMode = LensDiffSpectralMode.Spectral9
    p.wavelengthsNm = []
    p.rgbMode = LensDiffRgbMode.FromCaller
    return p, frame


def workload_zones8(seed: int = 1004):
    """The UHD 31-wavelength frame with field-varying aberrations on an 8 x 8
    zone grid, each zone its own PSF bank: coma and astigmatism grow with the
    normalised field radius (the reference's field model, a linear ramp with
    edge bias 0), their coefficients drawn ~N(0, 0.15) waves."""
    p, frame = workload_uhd31(seed)
    rng = np.random.default_rng(seed)
    coma_r, coma_t, astig_r, astig_t = (float(v) for v in rng.normal(0.0, 0.15, 4))
    p.phaseFieldStrength = 1.0
    p.phaseFieldEdgeBias = 0.0
    p.phaseFieldComaRadial = coma_r
    p.phaseFieldComaTangential = coma_t
    p.phaseFieldAstigRadial = astig_r
    p.phaseFieldAstigTangential = astig_t
    p.fieldGrid = 8
    return p, frame


def lens_instances(count: int = 256, seed: int = 1005, pupil=(128, 1024), pad=(2.0, 4.0), bins=(8, 64),
                   noll_max: int = 22) -> List[LensDiffParams]:
    """`count` unrelated lenses for batched bank builds: pupil N_p uniform in
    `pupil`, PSF size S = pad * N_p with pad uniform in `pad` (through the
    kernel radius R = pad * N_p / 4, since S = max(2 N_p, 512, 4 R)), B
    wavelengths uniform in `bins` spread over 400-700 nm with Gaussian RGB
    responses, 5-9 blade polygons with random rounding, obstruction and vanes,
    Noll 2..noll_max ~ N(0, 0.1) waves and chromatic focus 0.2 waves; the
    tensor-core (chosen) form."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        np_ = int(rng.integers(pupil[0], pupil[1] + 1))
        radius = max(4, int(round(float(rng.uniform(*pad)) * np_ / 4.0)))
        b = int(rng.integers(bins[0], bins[1] + 1))
        p = base_params(2160)
        p.apertureMode = LensDiffApertureMode.Polygon
        p.bladeCount = int(rng.integers(5, 10))
        p.roundness = float(rng.uniform(0.0, 1.0))
        p.centralObstruction = float(rng.choice([0.0, rng.uniform(0.1, 0.4)]))
        p.vaneCount = int(rng.integers(0, 5))
        p.vaneThickness = float(rng.uniform(0.005, 0.03))
        p.rotationDeg = float(rng.uniform(0.0, 60.0))
        p.pupilResolution = np_
        p.maxKernelRadiusPx = radius_percent(radius, 2160)
        noll = [0.0] * 23
        for j in range(2, noll_max + 1):
            noll[j] = float(rng.normal(0.0, 0.1))
        p.noll = noll
        p.chromaticFocus = 0.2
        p.spectralMode = LensDiffSpectralMode.Spectral9
        p.wavelengthsNm = [float(v) for v in np.linspace(400.0, 700.0, b)]
        p.rgbMode = LensDiffRgbMode.Gaussian
        p.fftForm = LensDiffFftForm.OwnChosen
        out.append(p)
    return out


def scaled_down(p: LensDiffParams, short_side: int, pupil: Optional[int] = None,
                max_radius_px: Optional[float] = None) -> LensDiffParams:
    """A smaller copy of a workload's lens for parity runs."""
    q = p.copy()
    q.frameShortSidePx = short_side
    if pupil is not None:
        q.pupilResolution = pupil
    if max_radius_px is not None:
        q.maxKernelRadiusPx = radius_percent(int(max_radius_px), short_side)
    return q
