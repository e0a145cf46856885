"""ctypes access to oracle/_ref/libldref.so — the reference's own CPU code,
compiled from its sources by oracle/Makefile.  TEST INFRASTRUCTURE ONLY."""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libldref.so")
# The reference project's source tree, named by the environment (the build
# script sets it where the sources are present; nothing here needs it at run time).
REF_ROOT = os.environ.get("LENSDIFF_REFERENCE_ROOT", "")

_lib: Optional[ctypes.CDLL] = None


def build(force: bool = False) -> bool:
    """Compiles the reference shim when the reference sources are present."""
    if os.path.exists(REF_LIB) and not force:
        return True
    if not REF_ROOT or not os.path.isdir(REF_ROOT):
        return False
    subprocess.run(["make", "-C", HERE, f"REF={REF_ROOT}"], check=True,
                   stdout=subprocess.DEVNULL)
    return os.path.exists(REF_LIB)


def available() -> bool:
    return os.path.exists(REF_LIB)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("oracle/_ref/libldref.so is not built")
        L = ctypes.CDLL(REF_LIB)
        fp = ctypes.POINTER(ctypes.c_float)
        ip = ctypes.POINTER(ctypes.c_int)
        vp = ctypes.c_void_p
        L.ldref_sizes.argtypes = [vp, ip, ip, ip]
        L.ldref_pupil.argtypes = [vp, fp, fp]
        L.ldref_raw_psf.argtypes = [vp, ctypes.c_float, fp]
        L.ldref_first_zero.argtypes = [ctypes.c_int, ctypes.c_int]
        L.ldref_first_zero.restype = ctypes.c_float
        L.ldref_first_zero_of.argtypes = [fp, ctypes.c_int]
        L.ldref_first_zero_of.restype = ctypes.c_float
        L.ldref_wavelengths.argtypes = [ctypes.c_int, fp]
        L.ldref_wavelengths.restype = ctypes.c_int
        L.ldref_bank.argtypes = [vp, fp, ip, fp, fp, fp, ctypes.c_longlong, ip]
        L.ldref_bank.restype = ctypes.c_int
        L.ldref_spectrum_config.argtypes = [vp, ctypes.c_int, fp, fp, fp]
        L.ldref_spectrum_config.restype = ctypes.c_int
        L.ldref_map_bins.argtypes = [vp, ctypes.c_int, fp, fp, ctypes.c_longlong, fp]
        L.ldref_render.argtypes = [vp, fp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   fp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_char_p, ctypes.c_int]
        L.ldref_render.restype = ctypes.c_int
        L.ldref_convolve_scalar.argtypes = [fp, ctypes.c_int, ctypes.c_int, fp, ctypes.c_int, fp]
        L.ldref_raw_psf_from.argtypes = [fp, fp, ctypes.c_int, ctypes.c_int, fp]
        L.ldref_resample.argtypes = [fp, ctypes.c_int, ctypes.c_float, ctypes.c_int, fp]
        _lib = L
    return _lib


def _f(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _abi(params):
    from lensdiff_b200.abi import to_abi_params
    s = to_abi_params(params)
    return s, ctypes.byref(s)


def sizes(params) -> Tuple[int, int, int]:
    s, ref = _abi(params)
    a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    lib().ldref_sizes(ref, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
    return a.value, b.value, c.value


def pupil(params):
    np_, _, _ = sizes(params)
    amp = np.zeros((np_, np_), np.float32)
    ph = np.zeros((np_, np_), np.float32)
    s, ref = _abi(params)
    lib().ldref_pupil(ref, _f(amp), _f(ph))
    return amp, ph


def raw_psf(params, wavelength: float = 550.0) -> np.ndarray:
    _, S, _ = sizes(params)
    out = np.zeros((S, S), np.float32)
    s, ref = _abi(params)
    lib().ldref_raw_psf(ref, float(wavelength), _f(out))
    return out


def raw_psf_from(pupil_amp: np.ndarray, phase: Optional[np.ndarray], size: int) -> np.ndarray:
    n = pupil_amp.shape[0]
    out = np.zeros((size, size), np.float32)
    a = np.ascontiguousarray(pupil_amp, np.float32)
    ph = None if phase is None else np.ascontiguousarray(phase, np.float32)
    lib().ldref_raw_psf_from(_f(a), None if ph is None else _f(ph), n, size, _f(out))
    return out


def first_zero(np_: int, size: int) -> float:
    return float(lib().ldref_first_zero(np_, size))


def resample(raw: np.ndarray, scale: float, radius: int) -> np.ndarray:
    k = 2 * radius + 1
    out = np.zeros((k, k), np.float32)
    r = np.ascontiguousarray(raw, np.float32)
    lib().ldref_resample(_f(r), r.shape[0], float(scale), int(radius), _f(out))
    return out


def bank(params):
    """Returns (wavelengths, [full], [core], [structure], support_radius)."""
    _, _, rmax = sizes(params)
    k = 2 * rmax + 1
    cap = 9 * k * k
    full = np.zeros(cap, np.float32)
    core = np.zeros(cap, np.float32)
    st = np.zeros(cap, np.float32)
    wl = np.zeros(9, np.float32)
    sz = (ctypes.c_int * 9)()
    sup = ctypes.c_int()
    s, ref = _abi(params)
    n = lib().ldref_bank(ref, _f(wl), sz, _f(full), _f(core), _f(st), cap, ctypes.byref(sup))
    if n < 0:
        raise RuntimeError("bank capacity")
    fulls, cores, sts = [], [], []
    off = 0
    for i in range(n):
        m = sz[i] * sz[i]
        fulls.append(full[off:off + m].reshape(sz[i], sz[i]).copy())
        cores.append(core[off:off + m].reshape(sz[i], sz[i]).copy())
        sts.append(st[off:off + m].reshape(sz[i], sz[i]).copy())
        off += m
    return [float(x) for x in wl[:n]], fulls, cores, sts, sup.value


def spectrum_matrices(params, wavelengths):
    """(natural 3xB, style 3xB) from BuildLensDiffSpectrumConfig."""
    wl = np.ascontiguousarray(wavelengths, np.float32)
    nat = np.zeros(27, np.float32)
    sty = np.zeros(27, np.float32)
    s, ref = _abi(params)
    cnt = lib().ldref_spectrum_config(ref, len(wl), _f(wl), _f(nat), _f(sty))
    b = len(wl)
    return nat.reshape(3, 9)[:, :b].copy(), sty.reshape(3, 9)[:, :b].copy(), cnt


def map_bins(params, wavelengths, values: np.ndarray) -> np.ndarray:
    wl = np.ascontiguousarray(wavelengths, np.float32)
    v = np.zeros((values.shape[0], 9), np.float32)
    v[:, : values.shape[1]] = values
    out = np.zeros((values.shape[0], 3), np.float32)
    s, ref = _abi(params)
    lib().ldref_map_bins(ref, len(wl), _f(wl), _f(v), values.shape[0], _f(out))
    return out


def render(params, src: np.ndarray, src_origin=(0, 0), dst_bounds=None, render_window=None):
    h, w = src.shape[:2]
    sx1, sy1 = src_origin
    if dst_bounds is None:
        dst_bounds = (sx1, sy1, sx1 + w, sy1 + h)
    if render_window is None:
        render_window = dst_bounds
    dx1, dy1, dx2, dy2 = dst_bounds
    dst = np.zeros((dy2 - dy1, dx2 - dx1, 4), np.float32)
    srcc = np.ascontiguousarray(src, np.float32)
    err = ctypes.create_string_buffer(256)
    s, ref = _abi(params)
    ok = lib().ldref_render(ref, _f(srcc), sx1, sy1, w, h, _f(dst), dx1, dy1, dx2 - dx1, dy2 - dy1,
                            render_window[0], render_window[1], render_window[2], render_window[3],
                            err, 256)
    if not ok:
        raise RuntimeError(err.value.decode())
    return dst


def convolve_scalar(plane: np.ndarray, kernel: np.ndarray) -> np.ndarray:
    h, w = plane.shape
    out = np.zeros((h, w), np.float32)
    p = np.ascontiguousarray(plane, np.float32)
    k = np.ascontiguousarray(kernel, np.float32)
    lib().ldref_convolve_scalar(_f(p), w, h, _f(k), k.shape[0], _f(out))
    return out


# ---------------------------------------------------------------------------
# The reference's own CUDA chain (oracle/_ref/libldrefcuda.so): the GPU
# comparator, RunLensDiffCuda of source/src/cuda/LensDiffCuda.cu on cuFFT.
# ---------------------------------------------------------------------------
REF_CUDA_LIB = os.path.join(HERE, "_ref", "libldrefcuda.so")
_cuda_lib: Optional[ctypes.CDLL] = None


def cuda_available() -> bool:
    return os.path.exists(REF_CUDA_LIB)


def cuda_lib() -> ctypes.CDLL:
    global _cuda_lib
    if _cuda_lib is None:
        if not cuda_available():
            raise RuntimeError("oracle/_ref/libldrefcuda.so is not built")
        L = ctypes.CDLL(REF_CUDA_LIB)
        vp = ctypes.c_void_p
        L.ldrefcuda_render.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, ctypes.c_longlong, vp, vp,
                                       ctypes.c_char_p, ctypes.c_int]
        L.ldrefcuda_render.restype = ctypes.c_int
        _cuda_lib = L
    return _cuda_lib


def cuda_render(params, src_ptr: int, dst_ptr: int, width: int, height: int, stream_ptr: int,
                instance: int = 0) -> None:
    """RunLensDiffCuda on device RGBA float buffers (rows of width * 16 bytes),
    enqueued on stream_ptr; `instance` picks one of four persistent
    LensDiffPsfBankCache objects, as the plugin keeps one per effect instance."""
    err = ctypes.create_string_buffer(256)
    s, ref = _abi(params)
    ok = cuda_lib().ldrefcuda_render(ref, int(instance), ctypes.c_void_p(src_ptr), int(width), int(height),
                                     int(width) * 16, ctypes.c_void_p(dst_ptr), ctypes.c_void_p(stream_ptr), err, 256)
    if not ok:
        raise RuntimeError("reference RunLensDiffCuda: " + err.value.decode())


def set_custom_aperture(values: np.ndarray, normalize: bool = True, invert: bool = False) -> None:
    """Hands a decoded amplitude image to the reference's own aperture loader
    (its cache), for the Custom aperture mode of later calls."""
    v = np.ascontiguousarray(values, np.float32)
    L = lib()
    L.ldref_set_custom_aperture.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_int]
    L.ldref_set_custom_aperture(_f(v), v.shape[1], v.shape[0], 1 if normalize else 0, 1 if invert else 0)
