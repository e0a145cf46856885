"""Host-side mirror of the reference's request / parameter types.

Field names, defaults and enum orders follow source/src/core/LensDiffTypes.h
(enums :14-91, LensDiffImageRect/View :94-111, LensDiffRenderRequest :113-126,
LensDiffParams :128-208) so that code written against the reference's C++ API
reads the same here.  The extension fields at the end of LensDiffParams (explicit
wavelength lists, Gaussian RGB responses, Noll terms outside 4..17, field grid
size, FFT form) default to values that keep the reference's behaviour.
"""
from __future__ import annotations

import dataclasses
import enum
from dataclasses import dataclass, field
from typing import Any, List, Optional

K_MAX_SPECTRAL_BINS = 9  # LensDiffTypes.h:12
MAX_WAVELENGTHS = 64
NOLL_COUNT = 23


class LensDiffExtractionMode(enum.IntEnum):
    MaxRgb = 0
    Luma = 1


class LensDiffApertureMode(enum.IntEnum):
    Circle = 0
    Polygon = 1
    Star = 2
    Spiral = 3
    Custom = 4
    Hexagon = 5
    SquareGrid = 6
    Snowflake = 7


class LensDiffApodizationMode(enum.IntEnum):
    Flat = 0
    Cosine = 1
    Gaussian = 2


class LensDiffSpectralMode(enum.IntEnum):
    Mono = 0
    Tristimulus = 1
    Spectral5 = 2
    Spectral9 = 3


class LensDiffSpectrumStyle(enum.IntEnum):
    Natural = 0
    CyanMagenta = 1
    WarmCool = 2


class LensDiffLookMode(enum.IntEnum):
    Physical = 0
    Split = 1


class LensDiffEnergyMode(enum.IntEnum):
    Preserve = 0
    Augment = 1


class LensDiffDebugView(enum.IntEnum):
    Final = 0
    Selection = 1
    Pupil = 2
    Psf = 3
    Otf = 4
    Core = 5
    Structure = 6
    Effect = 7
    Phase = 8
    PhaseEdge = 9
    FieldPsf = 10
    ChromaticSplit = 11
    CreativeFringe = 12
    Scatter = 13


class LensDiffInputTransfer(enum.IntEnum):
    Linear = 0
    DavinciIntermediate = 1


class LensDiffPhaseMode(enum.IntEnum):
    Off = 0
    Enabled = 1


class LensDiffRgbMode(enum.IntEnum):
    """Extension: where the spectral->RGB matrices come from."""
    FromCaller = 0
    Gaussian = 1


class LensDiffFftForm(enum.IntEnum):
    """Extension: which transform chain the device path uses."""
    OwnFp32 = 0
    OwnChosen = 1
    Cufft = 2


@dataclass
class LensDiffImageRect:
    x1: int = 0
    y1: int = 0
    x2: int = 0
    y2: int = 0

    def width(self) -> int:
        return self.x2 - self.x1

    def height(self) -> int:
        return self.y2 - self.y1


@dataclass
class LensDiffImageView:
    """`data` is a device address (int) or an object with data_ptr()."""
    data: object = None
    rowBytes: int = 0
    bounds: LensDiffImageRect = field(default_factory=LensDiffImageRect)
    originX: int = 0
    originY: int = 0
    components: int = 4
    bytesPerComponent: int = 4


@dataclass
class LensDiffRenderRequest:
    renderWindow: LensDiffImageRect = field(default_factory=LensDiffImageRect)
    frameBounds: LensDiffImageRect = field(default_factory=LensDiffImageRect)
    src: LensDiffImageView = field(default_factory=LensDiffImageView)
    dst: LensDiffImageView = field(default_factory=LensDiffImageView)
    frameShortSidePx: int = 0
    hostEnabledCudaRender: bool = False
    cudaStream: object = None  # int handle or torch.cuda.Stream


@dataclass
class LensDiffParams:
    extractionMode: LensDiffExtractionMode = LensDiffExtractionMode.MaxRgb
    apertureMode: LensDiffApertureMode = LensDiffApertureMode.Circle
    apodizationMode: LensDiffApodizationMode = LensDiffApodizationMode.Flat
    spectralMode: LensDiffSpectralMode = LensDiffSpectralMode.Mono
    spectrumStyle: LensDiffSpectrumStyle = LensDiffSpectrumStyle.Natural
    lookMode: LensDiffLookMode = LensDiffLookMode.Split
    energyMode: LensDiffEnergyMode = LensDiffEnergyMode.Preserve
    debugView: LensDiffDebugView = LensDiffDebugView.Final
    inputTransfer: LensDiffInputTransfer = LensDiffInputTransfer.Linear
    resolutionAware: bool = False

    threshold: float = 4.0
    softnessStops: float = 1.0
    pointEmphasis: float = 0.0
    corePreserve: float = 0.1

    bladeCount: int = 6
    roundness: float = 0.5
    rotationDeg: float = 0.0
    centralObstruction: float = 0.0
    vaneCount: int = 0
    vaneThickness: float = 0.01
    diffractionScalePx: float = 24.0
    pupilResolution: int = 256
    maxKernelRadiusPx: float = 64.0
    frameShortSidePx: int = 2160
    customAperturePath: str = ""
    customApertureNormalize: bool = True
    customApertureInvert: bool = False
    # Extension: the Custom aperture's image as the host decoded it (a 2-D
    # float array of amplitudes, rows first); the reference decodes
    # customAperturePath with WIC / ImageIO, which this machine has not.
    customApertureImage: Optional[Any] = None
    phaseMode: LensDiffPhaseMode = LensDiffPhaseMode.Off
    phaseDefocus: float = 0.0
    phaseAstigmatism0: float = 0.0
    phaseAstigmatism45: float = 0.0
    phaseComaX: float = 0.0
    phaseComaY: float = 0.0
    phaseSpherical: float = 0.0
    phaseTrefoilX: float = 0.0
    phaseTrefoilY: float = 0.0
    phaseSecondaryAstigmatism0: float = 0.0
    phaseSecondaryAstigmatism45: float = 0.0
    phaseQuadrafoil0: float = 0.0
    phaseQuadrafoil45: float = 0.0
    phaseSecondaryComaX: float = 0.0
    phaseSecondaryComaY: float = 0.0
    pupilDecenterX: float = 0.0
    pupilDecenterY: float = 0.0
    phaseFieldStrength: float = 0.0
    phaseFieldEdgeBias: float = 0.0
    phaseFieldDefocus: float = 0.0
    phaseFieldAstigRadial: float = 0.0
    phaseFieldAstigTangential: float = 0.0
    phaseFieldComaRadial: float = 0.0
    phaseFieldComaTangential: float = 0.0
    phaseFieldSpherical: float = 0.0
    phaseFieldTrefoilRadial: float = 0.0
    phaseFieldTrefoilTangential: float = 0.0
    phaseFieldSecondaryAstigRadial: float = 0.0
    phaseFieldSecondaryAstigTangential: float = 0.0
    phaseFieldQuadrafoilRadial: float = 0.0
    phaseFieldQuadrafoilTangential: float = 0.0
    phaseFieldSecondaryComaRadial: float = 0.0
    phaseFieldSecondaryComaTangential: float = 0.0

    spectrumForce: float = 0.0
    spectrumSaturation: float = 1.0
    chromaticAffectsLuma: bool = False
    chromaticFocus: float = 0.0
    chromaticSpread: float = 0.0
    creativeFringe: float = 0.0
    scatterAmount: float = 0.0
    scatterRadius: float = 0.0

    effectGain: float = 1.0
    coreCompensation: float = 1.0
    anisotropyEmphasis: float = 0.0
    coreGain: float = 1.0
    structureGain: float = 1.0
    coreShoulder: float = 0.0
    structureShoulder: float = 0.0

    # ---- extensions (defaults keep the reference's behaviour) ----------
    wavelengthsNm: Optional[List[float]] = None      # None: spectralMode's set
    rgbMode: LensDiffRgbMode = LensDiffRgbMode.FromCaller
    naturalMatrix: Optional[List[List[float]]] = None  # 3 x B
    styleMatrix: Optional[List[List[float]]] = None    # 3 x B
    rgbGaussCenterNm: tuple = (600.0, 540.0, 450.0)
    rgbGaussSigmaNm: float = 40.0
    noll: Optional[List[float]] = None                 # index j = 0..22
    fieldGrid: int = 0
    fftForm: LensDiffFftForm = LensDiffFftForm.OwnFp32

    def copy(self, **changes) -> "LensDiffParams":
        return dataclasses.replace(self, **changes)


# Wavelength sets of the reference spectral modes (LensDiffCpuReference.cpp:1602-1614).
SPECTRAL_MODE_WAVELENGTHS = {
    LensDiffSpectralMode.Mono: [550.0],
    LensDiffSpectralMode.Tristimulus: [460.0, 550.0, 610.0],
    LensDiffSpectralMode.Spectral5: [440.0, 490.0, 540.0, 590.0, 640.0],
    LensDiffSpectralMode.Spectral9: [420.0, 450.0, 480.0, 510.0, 540.0, 570.0, 600.0, 630.0, 660.0],
}


def resolved_wavelengths(params: LensDiffParams) -> List[float]:
    if params.wavelengthsNm:
        return [float(w) for w in params.wavelengthsNm]
    return list(SPECTRAL_MODE_WAVELENGTHS[LensDiffSpectralMode(params.spectralMode)])
