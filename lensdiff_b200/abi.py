"""ctypes mirror of include/lensdiff_b200.h and the loader of the native library.

The structures here must match the header field for field; a CPU test checks
their sizes against the C compiler's (tests/test_abi.py).  The library is
loaded from this package directory (built in place by lensdiff_b200.build);
if it is missing the import of `lib()` raises — there is no fallback.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

from .types import (
    MAX_WAVELENGTHS,
    NOLL_COUNT,
    LensDiffParams,
    LensDiffRgbMode,
    LensDiffSpectralMode,
    resolved_wavelengths,
)

LIB_NAME = "liblensdiff_b200.so"
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)

LD_OK = 0
LD_ERR_ARG = 1
LD_ERR_OOM = 2
LD_ERR_BUDGET = 3
LD_ERR_TIMEOUT = 4
LD_ERR_CUDA = 5
LD_ERR_UNSUPPORTED = 6
STAGE_LEN = 128

c_i32 = ctypes.c_int32
c_f64 = ctypes.c_double
c_f32 = ctypes.c_float


class ld_rect(ctypes.Structure):
    _fields_ = [("x1", c_i32), ("y1", c_i32), ("x2", c_i32), ("y2", c_i32)]


class ld_image_view(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.c_void_p),
        ("row_bytes", ctypes.c_int64),
        ("bounds", ld_rect),
        ("origin_x", c_i32),
        ("origin_y", c_i32),
        ("components", c_i32),
        ("bytes_per_component", c_i32),
    ]


class ld_render_request(ctypes.Structure):
    _fields_ = [
        ("render_window", ld_rect),
        ("frame_bounds", ld_rect),
        ("src", ld_image_view),
        ("dst", ld_image_view),
        ("frame_short_side_px", c_i32),
        ("host_enabled_cuda_render", c_i32),
        ("cuda_stream", ctypes.c_void_p),
    ]


_PARAM_FIELDS = [
    ("extraction_mode", c_i32),
    ("aperture_mode", c_i32),
    ("apodization_mode", c_i32),
    ("spectral_mode", c_i32),
    ("spectrum_style", c_i32),
    ("look_mode", c_i32),
    ("energy_mode", c_i32),
    ("debug_view", c_i32),
    ("input_transfer", c_i32),
    ("resolution_aware", c_i32),
    ("threshold", c_f64),
    ("softness_stops", c_f64),
    ("point_emphasis", c_f64),
    ("core_preserve", c_f64),
    ("blade_count", c_i32),
    ("vane_count", c_i32),
    ("roundness", c_f64),
    ("rotation_deg", c_f64),
    ("central_obstruction", c_f64),
    ("vane_thickness", c_f64),
    ("diffraction_scale_px", c_f64),
    ("pupil_resolution", c_i32),
    ("frame_short_side_px", c_i32),
    ("max_kernel_radius_px", c_f64),
    ("phase_mode", c_i32),
    ("chromatic_affects_luma", c_i32),
    ("phase_defocus", c_f64),
    ("phase_astigmatism0", c_f64),
    ("phase_astigmatism45", c_f64),
    ("phase_coma_x", c_f64),
    ("phase_coma_y", c_f64),
    ("phase_spherical", c_f64),
    ("phase_trefoil_x", c_f64),
    ("phase_trefoil_y", c_f64),
    ("phase_secondary_astigmatism0", c_f64),
    ("phase_secondary_astigmatism45", c_f64),
    ("phase_quadrafoil0", c_f64),
    ("phase_quadrafoil45", c_f64),
    ("phase_secondary_coma_x", c_f64),
    ("phase_secondary_coma_y", c_f64),
    ("pupil_decenter_x", c_f64),
    ("pupil_decenter_y", c_f64),
    ("phase_field_strength", c_f64),
    ("phase_field_edge_bias", c_f64),
    ("phase_field_defocus", c_f64),
    ("phase_field_astig_radial", c_f64),
    ("phase_field_astig_tangential", c_f64),
    ("phase_field_coma_radial", c_f64),
    ("phase_field_coma_tangential", c_f64),
    ("phase_field_spherical", c_f64),
    ("phase_field_trefoil_radial", c_f64),
    ("phase_field_trefoil_tangential", c_f64),
    ("phase_field_secondary_astig_radial", c_f64),
    ("phase_field_secondary_astig_tangential", c_f64),
    ("phase_field_quadrafoil_radial", c_f64),
    ("phase_field_quadrafoil_tangential", c_f64),
    ("phase_field_secondary_coma_radial", c_f64),
    ("phase_field_secondary_coma_tangential", c_f64),
    ("spectrum_force", c_f64),
    ("spectrum_saturation", c_f64),
    ("chromatic_focus", c_f64),
    ("chromatic_spread", c_f64),
    ("creative_fringe", c_f64),
    ("scatter_amount", c_f64),
    ("scatter_radius", c_f64),
    ("effect_gain", c_f64),
    ("core_compensation", c_f64),
    ("anisotropy_emphasis", c_f64),
    ("core_gain", c_f64),
    ("structure_gain", c_f64),
    ("core_shoulder", c_f64),
    ("structure_shoulder", c_f64),
    ("wavelength_count", c_i32),
    ("wavelengths_nm", c_f32 * MAX_WAVELENGTHS),
    ("rgb_mode", c_i32),
    ("field_grid", c_i32),
    ("natural_matrix", c_f32 * (3 * MAX_WAVELENGTHS)),
    ("style_matrix", c_f32 * (3 * MAX_WAVELENGTHS)),
    ("rgb_gauss_center_nm", c_f32 * 3),
    ("rgb_gauss_sigma_nm", c_f32),
    ("noll", c_f64 * NOLL_COUNT),
    ("fft_form", c_i32),
    ("reserved", c_i32 * 7),
]


class ld_params(ctypes.Structure):
    _fields_ = _PARAM_FIELDS


class ld_status(ctypes.Structure):
    _fields_ = [
        ("code", c_i32),
        ("stage", ctypes.c_char * STAGE_LEN),
        ("bank_rebuilt", c_i32),
        ("spectra_rebuilt", c_i32),
        ("pupil_size", c_i32),
        ("raw_psf_size", c_i32),
        ("max_kernel_radius", c_i32),
        ("support_radius", c_i32),
        ("grid_requested_w", c_i32),
        ("grid_requested_h", c_i32),
        ("grid_used_w", c_i32),
        ("grid_used_h", c_i32),
        ("wavelength_count", c_i32),
        ("kernel_launches", c_i32),
    ]


# Reference camelCase name -> ABI snake_case name, for the scalar fields.
_SCALAR_MAP = {
    "extractionMode": "extraction_mode",
    "apertureMode": "aperture_mode",
    "apodizationMode": "apodization_mode",
    "spectralMode": "spectral_mode",
    "spectrumStyle": "spectrum_style",
    "lookMode": "look_mode",
    "energyMode": "energy_mode",
    "debugView": "debug_view",
    "inputTransfer": "input_transfer",
    "resolutionAware": "resolution_aware",
    "threshold": "threshold",
    "softnessStops": "softness_stops",
    "pointEmphasis": "point_emphasis",
    "corePreserve": "core_preserve",
    "bladeCount": "blade_count",
    "vaneCount": "vane_count",
    "roundness": "roundness",
    "rotationDeg": "rotation_deg",
    "centralObstruction": "central_obstruction",
    "vaneThickness": "vane_thickness",
    "diffractionScalePx": "diffraction_scale_px",
    "pupilResolution": "pupil_resolution",
    "frameShortSidePx": "frame_short_side_px",
    "maxKernelRadiusPx": "max_kernel_radius_px",
    "phaseMode": "phase_mode",
    "chromaticAffectsLuma": "chromatic_affects_luma",
    "phaseDefocus": "phase_defocus",
    "phaseAstigmatism0": "phase_astigmatism0",
    "phaseAstigmatism45": "phase_astigmatism45",
    "phaseComaX": "phase_coma_x",
    "phaseComaY": "phase_coma_y",
    "phaseSpherical": "phase_spherical",
    "phaseTrefoilX": "phase_trefoil_x",
    "phaseTrefoilY": "phase_trefoil_y",
    "phaseSecondaryAstigmatism0": "phase_secondary_astigmatism0",
    "phaseSecondaryAstigmatism45": "phase_secondary_astigmatism45",
    "phaseQuadrafoil0": "phase_quadrafoil0",
    "phaseQuadrafoil45": "phase_quadrafoil45",
    "phaseSecondaryComaX": "phase_secondary_coma_x",
    "phaseSecondaryComaY": "phase_secondary_coma_y",
    "pupilDecenterX": "pupil_decenter_x",
    "pupilDecenterY": "pupil_decenter_y",
    "phaseFieldStrength": "phase_field_strength",
    "phaseFieldEdgeBias": "phase_field_edge_bias",
    "phaseFieldDefocus": "phase_field_defocus",
    "phaseFieldAstigRadial": "phase_field_astig_radial",
    "phaseFieldAstigTangential": "phase_field_astig_tangential",
    "phaseFieldComaRadial": "phase_field_coma_radial",
    "phaseFieldComaTangential": "phase_field_coma_tangential",
    "phaseFieldSpherical": "phase_field_spherical",
    "phaseFieldTrefoilRadial": "phase_field_trefoil_radial",
    "phaseFieldTrefoilTangential": "phase_field_trefoil_tangential",
    "phaseFieldSecondaryAstigRadial": "phase_field_secondary_astig_radial",
    "phaseFieldSecondaryAstigTangential": "phase_field_secondary_astig_tangential",
    "phaseFieldQuadrafoilRadial": "phase_field_quadrafoil_radial",
    "phaseFieldQuadrafoilTangential": "phase_field_quadrafoil_tangential",
    "phaseFieldSecondaryComaRadial": "phase_field_secondary_coma_radial",
    "phaseFieldSecondaryComaTangential": "phase_field_secondary_coma_tangential",
    "spectrumForce": "spectrum_force",
    "spectrumSaturation": "spectrum_saturation",
    "chromaticFocus": "chromatic_focus",
    "chromaticSpread": "chromatic_spread",
    "creativeFringe": "creative_fringe",
    "scatterAmount": "scatter_amount",
    "scatterRadius": "scatter_radius",
    "effectGain": "effect_gain",
    "coreCompensation": "core_compensation",
    "anisotropyEmphasis": "anisotropy_emphasis",
    "coreGain": "core_gain",
    "structureGain": "structure_gain",
    "coreShoulder": "core_shoulder",
    "structureShoulder": "structure_shoulder",
}


def to_abi_params(p: LensDiffParams) -> ld_params:
    """Packs a LensDiffParams into the C struct (a field-by-field copy)."""
    out = ld_params()
    for src, dst in _SCALAR_MAP.items():
        v = getattr(p, src)
        ftype = dict(_PARAM_FIELDS)[dst]
        setattr(out, dst, int(v) if ftype is c_i32 else float(v))
    if p.wavelengthsNm:
        w = list(p.wavelengthsNm)
        if len(w) > MAX_WAVELENGTHS:
            raise ValueError(f"at most {MAX_WAVELENGTHS} wavelengths")
        out.wavelength_count = len(w)
        for i, x in enumerate(w):
            out.wavelengths_nm[i] = float(x)
    out.rgb_mode = int(p.rgbMode)
    out.field_grid = int(p.fieldGrid)
    nb = len(resolved_wavelengths(p))
    for name, mat in (("natural_matrix", p.naturalMatrix), ("style_matrix", p.styleMatrix)):
        if mat is not None:
            arr = getattr(out, name)
            for r in range(3):
                if len(mat[r]) < nb:
                    raise ValueError(f"{name} row {r} needs {nb} entries")
                for b in range(nb):
                    arr[r * nb + b] = float(mat[r][b])
    for i in range(3):
        out.rgb_gauss_center_nm[i] = float(p.rgbGaussCenterNm[i])
    out.rgb_gauss_sigma_nm = float(p.rgbGaussSigmaNm)
    if p.noll is not None:
        for j, v in enumerate(p.noll[:NOLL_COUNT]):
            out.noll[j] = float(v)
    out.fft_form = int(p.fftForm)
    return out


_LIB: Optional[ctypes.CDLL] = None

EXPORTED_SYMBOLS = [
    "ld_create",
    "ld_destroy",
    "ld_abi_version",
    "ld_device_bytes",
    "ld_clear_caches",
    "ld_check_device_errors",
    "ld_render",
    "ld_build_psf_bank",
    "ld_build_psf_banks",
    "ld_profile_tensor_flops",
    "ld_export_psf_bank",
    "ld_raw_psf",
    "ld_raw_psf_noalloc",
    "ld_resolve_sizes",
    "ld_gaussian_rgb_matrix",
    "ld_set_profiling",
    "ld_profile_collect",
    "ld_estimate_device_bytes",
    "ld_set_graphs",
    "ld_set_autotune",
    "ld_selftest_wait",
    "ld_set_custom_aperture",
    "ld_export_kernel_spectra",
    "ld_import_kernel_spectra",
    "ld_inject_alloc_failure",
    "ld_autotune_choice",
    "ld_server_create",
    "ld_server_destroy",
    "ld_server_submit",
    "ld_server_wait",
    "ld_server_get_stats",
    "ld_server_reset_stats",
]


class ld_server_stats(ctypes.Structure):
    _fields_ = [
        ("completed", ctypes.c_uint64), ("pending", ctypes.c_uint64), ("cache_hits", ctypes.c_uint64),
        ("max_concurrent", ctypes.c_uint64), ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
        ("mean_ms", ctypes.c_double), ("frames_per_s", ctypes.c_double), ("device_bytes", ctypes.c_size_t),
        ("reserved_bytes", ctypes.c_size_t),
    ]

STAGE_NAMES = ["psf_rows", "psf_cols", "resample", "shape_stats", "support", "crop_sum", "combine",
               "kspec_rows", "kspec_cols", "frame_rows", "frame_cols", "frame_inverse", "pupil", "composite",
               "scatter", "working_source", "dft_gemm"]


def lib() -> ctypes.CDLL:
    """Loads liblensdiff_b200.so from the package directory (no fallback)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_NAME} is not built; run `python -m lensdiff_b200.build` "
            "(the CUDA path has no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    L.ld_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_size_t]
    L.ld_create.restype = ctypes.c_int
    L.ld_destroy.argtypes = [vp]
    L.ld_destroy.restype = None
    L.ld_abi_version.argtypes = []
    L.ld_abi_version.restype = ctypes.c_int
    L.ld_device_bytes.argtypes = [vp]
    L.ld_device_bytes.restype = ctypes.c_size_t
    L.ld_clear_caches.argtypes = [vp]
    L.ld_clear_caches.restype = None
    L.ld_render.argtypes = [vp, ctypes.POINTER(ld_render_request), ctypes.POINTER(ld_params),
                            ctypes.POINTER(ld_status)]
    L.ld_render.restype = ctypes.c_int
    L.ld_build_psf_bank.argtypes = [vp, ctypes.POINTER(ld_params), vp, ctypes.POINTER(ld_status)]
    L.ld_build_psf_bank.restype = ctypes.c_int
    L.ld_build_psf_banks.argtypes = [vp, ctypes.POINTER(ld_params), ctypes.c_int32, vp, ctypes.POINTER(ld_status)]
    L.ld_build_psf_banks.restype = ctypes.c_int
    L.ld_profile_tensor_flops.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
    L.ld_profile_tensor_flops.restype = ctypes.c_int
    L.ld_export_psf_bank.argtypes = [vp, ctypes.POINTER(ld_params), vp,
                                     ctypes.POINTER(c_f32), ctypes.POINTER(c_i32),
                                     ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(c_f32),
                                     ctypes.c_int64, ctypes.POINTER(ld_status)]
    L.ld_export_psf_bank.restype = ctypes.c_int
    L.ld_raw_psf.argtypes = [vp, ctypes.POINTER(ld_params), ctypes.c_int, vp, vp,
                             ctypes.POINTER(ld_status)]
    L.ld_raw_psf.restype = ctypes.c_int
    L.ld_raw_psf_noalloc.argtypes = [ctypes.POINTER(ld_params), ctypes.c_int, vp, vp, ctypes.POINTER(ld_status)]
    L.ld_raw_psf_noalloc.restype = ctypes.c_int
    L.ld_resolve_sizes.argtypes = [ctypes.POINTER(ld_params), ctypes.POINTER(c_i32),
                                   ctypes.POINTER(c_i32), ctypes.POINTER(c_i32),
                                   ctypes.POINTER(c_i32)]
    L.ld_resolve_sizes.restype = ctypes.c_int
    L.ld_gaussian_rgb_matrix.argtypes = [ctypes.POINTER(c_f32), c_i32, ctypes.POINTER(c_f32),
                                         c_f32, ctypes.POINTER(c_f32)]
    L.ld_gaussian_rgb_matrix.restype = ctypes.c_int
    L.ld_check_device_errors.argtypes = [vp, ctypes.POINTER(c_i32)]
    L.ld_check_device_errors.restype = ctypes.c_int
    L.ld_set_profiling.argtypes = [vp, ctypes.c_int]
    L.ld_set_profiling.restype = ctypes.c_int
    L.ld_profile_collect.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(c_i32), c_i32]
    L.ld_profile_collect.restype = ctypes.c_int
    L.ld_set_graphs.argtypes = [vp, ctypes.c_int]
    L.ld_set_graphs.restype = ctypes.c_int
    L.ld_export_kernel_spectra.argtypes = [vp, ctypes.POINTER(ld_params), c_i32, c_i32, vp, ctypes.c_size_t,
                                           ctypes.POINTER(ctypes.c_size_t), vp, ctypes.POINTER(ld_status)]
    L.ld_export_kernel_spectra.restype = ctypes.c_int
    L.ld_import_kernel_spectra.argtypes = [vp, ctypes.POINTER(ld_params), c_i32, c_i32, vp, ctypes.c_size_t, vp,
                                           ctypes.POINTER(ld_status)]
    L.ld_import_kernel_spectra.restype = ctypes.c_int
    L.ld_set_custom_aperture.argtypes = [vp, ctypes.POINTER(c_f32), c_i32, c_i32, c_i32, c_i32]
    L.ld_set_custom_aperture.restype = ctypes.c_int
    L.ld_selftest_wait.argtypes = [vp, c_i32, ctypes.c_int64, vp, ctypes.POINTER(c_i32)]
    L.ld_selftest_wait.restype = ctypes.c_int
    L.ld_inject_alloc_failure.argtypes = [vp, c_i32]
    L.ld_inject_alloc_failure.restype = ctypes.c_int
    L.ld_set_autotune.argtypes = [vp, ctypes.c_int]
    L.ld_set_autotune.restype = ctypes.c_int
    L.ld_autotune_choice.argtypes = [vp, c_i32, ctypes.POINTER(c_i32), ctypes.POINTER(c_i32),
                                     ctypes.POINTER(ctypes.c_double)]
    L.ld_autotune_choice.restype = ctypes.c_int
    L.ld_estimate_device_bytes.argtypes = [ctypes.POINTER(ld_params), c_i32, c_i32]
    L.ld_estimate_device_bytes.restype = ctypes.c_size_t
    L.ld_server_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int, ctypes.c_size_t]
    L.ld_server_create.restype = ctypes.c_int
    L.ld_server_destroy.argtypes = [vp]
    L.ld_server_destroy.restype = None
    L.ld_server_submit.argtypes = [vp, vp, vp, c_i32, c_i32, ctypes.POINTER(ld_params),
                                   ctypes.POINTER(ctypes.c_uint64)]
    L.ld_server_submit.restype = ctypes.c_int
    L.ld_server_wait.argtypes = [vp, ctypes.c_uint64, ctypes.c_double, ctypes.POINTER(ld_status),
                                 ctypes.POINTER(ctypes.c_double)]
    L.ld_server_wait.restype = ctypes.c_int
    L.ld_server_get_stats.argtypes = [vp, ctypes.POINTER(ld_server_stats)]
    L.ld_server_get_stats.restype = ctypes.c_int
    L.ld_server_reset_stats.argtypes = [vp]
    L.ld_server_reset_stats.restype = None
    if L.ld_abi_version() != 1:
        raise RuntimeError("liblensdiff_b200.so ABI version mismatch")
    _LIB = L
    return L


def is_spectral(p: LensDiffParams) -> bool:
    return len(resolved_wavelengths(p)) > 1 or (
        p.wavelengthsNm is None and LensDiffSpectralMode(p.spectralMode) != LensDiffSpectralMode.Mono)


__all__ = [
    "ld_rect", "ld_image_view", "ld_render_request", "ld_params", "ld_status",
    "to_abi_params", "lib", "LIB_PATH", "EXPORTED_SYMBOLS", "LensDiffRgbMode", "ld_server_stats",
]
