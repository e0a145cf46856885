"""Host-side mirror of the reference's CUDA backend entry point.

`run_lensdiff_cuda(request, params, cache, error)` has the meaning and error
behaviour of

    bool RunLensDiffCuda(const LensDiffRenderRequest& request,
                         const LensDiffParams& params,
                         LensDiffPsfBankCache& cache,
                         std::string* error);

(source/src/cuda/LensDiffCuda.h:7-10): it returns True on success, False with a
stage string on failure, and never falls back to a CPU path.  The PSF-bank
cache is device resident and owned by a `LensDiffPsfBankCache` (one per effect
instance, as the plugin keeps one `cache_` per instance, LensDiff.cpp:3833).

Everything here is a thin ctypes layer over liblensdiff_b200.so; device memory
is addressed by integer pointers (torch tensors are accepted and their
data_ptr() used).
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import abi
from .types import (
    LensDiffImageRect,
    LensDiffImageView,
    LensDiffParams,
    LensDiffRenderRequest,
)


def _ptr(x) -> Optional[int]:
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return int(x.data_ptr())
    raise TypeError(f"cannot take a device address of {type(x)!r}")


def _stream(x) -> Optional[int]:
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "cuda_stream"):
        return int(x.cuda_stream)
    raise TypeError(f"cannot take a stream handle of {type(x)!r}")


def _rect(r: LensDiffImageRect) -> abi.ld_rect:
    return abi.ld_rect(int(r.x1), int(r.y1), int(r.x2), int(r.y2))


def _view(v: LensDiffImageView) -> abi.ld_image_view:
    out = abi.ld_image_view()
    p = _ptr(v.data)
    out.data = p if p else None
    out.row_bytes = int(v.rowBytes)
    out.bounds = _rect(v.bounds)
    out.origin_x = int(v.originX)
    out.origin_y = int(v.originY)
    out.components = int(v.components)
    out.bytes_per_component = int(v.bytesPerComponent)
    return out


def to_abi_request(r: LensDiffRenderRequest) -> abi.ld_render_request:
    out = abi.ld_render_request()
    out.render_window = _rect(r.renderWindow)
    out.frame_bounds = _rect(r.frameBounds)
    out.src = _view(r.src)
    out.dst = _view(r.dst)
    out.frame_short_side_px = int(r.frameShortSidePx)
    out.host_enabled_cuda_render = 1 if r.hostEnabledCudaRender else 0
    s = _stream(r.cudaStream)
    out.cuda_stream = s if s else None
    return out


class LensDiffStatus:
    def __init__(self, st: abi.ld_status):
        self.code = int(st.code)
        self.stage = st.stage.decode(errors="replace")
        self.bank_rebuilt = bool(st.bank_rebuilt)
        self.banks_rebuilt = int(st.bank_rebuilt)  # lens sets: the banks built
        self.spectra_rebuilt = bool(st.spectra_rebuilt)
        self.pupil_size = int(st.pupil_size)
        self.raw_psf_size = int(st.raw_psf_size)
        self.max_kernel_radius = int(st.max_kernel_radius)
        self.support_radius = int(st.support_radius)
        self.grid_requested = (int(st.grid_requested_w), int(st.grid_requested_h))
        self.grid_used = (int(st.grid_used_w), int(st.grid_used_h))
        self.wavelength_count = int(st.wavelength_count)
        self.kernel_launches = int(st.kernel_launches)

    @property
    def ok(self) -> bool:
        return self.code == abi.LD_OK

    def __repr__(self) -> str:
        return f"LensDiffStatus(code={self.code}, stage={self.stage!r}, grid_used={self.grid_used})"


class LensDiffPsfBankCache:
    """Device-resident PSF-bank / kernel-spectrum cache of one effect instance
    (the B200 counterpart of LensDiffPsfBankCache, LensDiffTypes.h:396-412)."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self._lib = abi.lib()
        h = ctypes.c_void_p()
        rc = self._lib.ld_create(ctypes.byref(h), int(device), int(hbm_budget_bytes))
        if rc != abi.LD_OK:
            raise RuntimeError(f"ld_create failed with code {rc}")
        self._h = h
        self.device = device

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def close(self) -> None:
        if self._h:
            self._lib.ld_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def device_bytes(self) -> int:
        return int(self._lib.ld_device_bytes(self._h))

    def clear(self) -> None:
        self._lib.ld_clear_caches(self._h)

    def check_device_errors(self) -> int:
        """Reads and clears the device error word: 0 none, 1 a bulk-copy wait ran
        out of time, 2 a bulk copy failed its alignment / bounds check."""
        w = ctypes.c_int32()
        self._lib.ld_check_device_errors(self._h, ctypes.byref(w))
        return int(w.value)

    def set_graphs(self, enable: bool) -> None:
        """Replay per-frame chains as CUDA graphs (default on)."""
        self._lib.ld_set_graphs(self._h, 1 if enable else 0)

    def set_autotune(self, mode: int) -> None:
        """1: time the compiled radix orders of a new grid's transform lengths
        on its first composite frame and keep the fastest (the default); 0: the
        first compiled order; 2 + k: the k-th compiled order of each length
        (its last when it has fewer); -1: runtime-planned transforms only."""
        rc = self._lib.ld_set_autotune(self._h, int(mode))
        if rc != abi.LD_OK:
            raise ValueError(f"autotune mode {mode!r} rejected ({rc})")

    def autotune_choice(self, n: int):
        """(radix order, launch shape, ms) the autotuner chose for transform
        length n, or None."""
        r = (abi.c_i32 * 4)()
        shape = abi.c_i32(0)
        ms = ctypes.c_double(0.0)
        k = self._lib.ld_autotune_choice(self._h, int(n), r, ctypes.byref(shape), ctypes.byref(ms))
        return (tuple(int(r[i]) for i in range(k)), int(shape.value), float(ms.value)) if k else None

    def set_profiling(self, enable: bool) -> None:
        self._lib.ld_set_profiling(self._h, 1 if enable else 0)

    def profile_collect(self) -> dict:
        """{stage name: (device ms summed, launches)} since the last collect."""
        n = len(abi.STAGE_NAMES)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_int32 * n)()
        self._lib.ld_profile_collect(self._h, ms, cnt, n)
        return {abi.STAGE_NAMES[i]: (float(ms[i]), int(cnt[i])) for i in range(n)}

    def tensor_flops(self) -> float:
        """Tensor-core MMA flops issued by DFT-GEMM launches since the last call."""
        f = ctypes.c_double(0.0)
        self._lib.ld_profile_tensor_flops(self._h, ctypes.byref(f))
        return float(f.value)

    # -- entry points -------------------------------------------------------
    def set_custom_aperture(self, image, normalize: bool = True, invert: bool = False) -> int:
        """Hands the Custom aperture's decoded amplitude image (2-D, rows
        first) to the context (ld_set_custom_aperture); None clears it."""
        if image is None:
            self._custom_key = None
            return self._lib.ld_set_custom_aperture(self._h, None, 0, 0, 0, 0)
        a = np.ascontiguousarray(image, dtype=np.float32)
        if a.ndim != 2:
            raise ValueError("the custom aperture image must be 2-D")
        rc = self._lib.ld_set_custom_aperture(self._h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                              a.shape[1], a.shape[0], 1 if normalize else 0, 1 if invert else 0)
        self._custom_key = (a.shape, a.tobytes(), bool(normalize), bool(invert)) if rc == abi.LD_OK else None
        return rc

    def _sync_custom(self, params: LensDiffParams) -> None:
        img = getattr(params, "customApertureImage", None)
        if int(params.apertureMode) != 4 or img is None:
            return
        a = np.ascontiguousarray(img, dtype=np.float32)
        key = (a.shape, a.tobytes(), bool(params.customApertureNormalize), bool(params.customApertureInvert))
        if getattr(self, "_custom_key", None) != key:
            self.set_custom_aperture(a, params.customApertureNormalize, params.customApertureInvert)

    def render(self, request: LensDiffRenderRequest, params: LensDiffParams) -> LensDiffStatus:
        self._sync_custom(params)
        rq = to_abi_request(request)
        pp = abi.to_abi_params(params)
        st = abi.ld_status()
        self._lib.ld_render(self._h, ctypes.byref(rq), ctypes.byref(pp), ctypes.byref(st))
        return LensDiffStatus(st)

    def build_psf_bank(self, params: LensDiffParams, stream=None) -> LensDiffStatus:
        self._sync_custom(params)
        pp = abi.to_abi_params(params)
        st = abi.ld_status()
        self._lib.ld_build_psf_bank(self._h, ctypes.byref(pp), _stream(stream), ctypes.byref(st))
        return LensDiffStatus(st)

    def kernel_spectra_bytes(self, params: LensDiffParams, width: int, height: int) -> Tuple[int, LensDiffStatus]:
        """Size of the kernel-spectra block of a lens for a width x height frame."""
        pp = abi.to_abi_params(params)
        st = abi.ld_status()
        n = ctypes.c_size_t(0)
        self._lib.ld_export_kernel_spectra(self._h, ctypes.byref(pp), int(width), int(height), None, 0,
                                           ctypes.byref(n), None, ctypes.byref(st))
        return int(n.value), LensDiffStatus(st)

    def export_kernel_spectra(self, params: LensDiffParams, width: int, height: int, out, stream=None) -> LensDiffStatus:
        """Builds (if needed) and copies the kernel spectra into the device buffer `out`."""
        pp = abi.to_abi_params(params)
        st = abi.ld_status()
        n = ctypes.c_size_t(0)
        cap = int(out.numel() * out.element_size()) if hasattr(out, "numel") else 0
        self._lib.ld_export_kernel_spectra(self._h, ctypes.byref(pp), int(width), int(height), _ptr(out), cap,
                                           ctypes.byref(n), _stream(stream), ctypes.byref(st))
        return LensDiffStatus(st)

    def import_kernel_spectra(self, params: LensDiffParams, width: int, height: int, src, nbytes: int,
                              stream=None) -> LensDiffStatus:
        """Installs kernel spectra exported by another context for the same lens and frame size."""
        pp = abi.to_abi_params(params)
        st = abi.ld_status()
        self._lib.ld_import_kernel_spectra(self._h, ctypes.byref(pp), int(width), int(height), _ptr(src), int(nbytes),
                                           _stream(stream), ctypes.byref(st))
        return LensDiffStatus(st)

    def build_psf_banks(self, params_list: Sequence[LensDiffParams], stream=None) -> LensDiffStatus:
        """Builds the banks of several unrelated lenses together (their
        tensor-core windows in one launch per transform pass); they stay
        cached until the next call, for export_psf_bank and render."""
        arr = (abi.ld_params * len(params_list))()
        for i, p in enumerate(params_list):
            arr[i] = abi.to_abi_params(p)
        st = abi.ld_status()
        self._lib.ld_build_psf_banks(self._h, arr, len(params_list), _stream(stream), ctypes.byref(st))
        return LensDiffStatus(st)

    def export_psf_bank(self, params: LensDiffParams, stream=None) -> Tuple[List[float], List[np.ndarray], LensDiffStatus]:
        """Host copies of the bank's `full` kernels (one per wavelength)."""
        self._sync_custom(params)
        pp = abi.to_abi_params(params)
        np_, S, R, B = resolve_sizes(params)
        k = 2 * R + 1
        cap = B * k * k
        wl = np.zeros(B, np.float32)
        sizes = np.zeros(B, np.int32)
        offs = np.zeros(B, np.int64)
        buf = np.zeros(cap, np.float32)
        st = abi.ld_status()
        self._lib.ld_export_psf_bank(
            self._h, ctypes.byref(pp), _stream(stream),
            wl.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
            sizes.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
            offs.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
            buf.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), cap, ctypes.byref(st))
        status = LensDiffStatus(st)
        kernels = []
        if status.ok:
            for i in range(B):
                n = int(sizes[i])
                kernels.append(buf[offs[i]: offs[i] + n * n].reshape(n, n).copy())
        return [float(x) for x in wl], kernels, status

    def raw_psf(self, params: LensDiffParams, wavelength_index: int, out, stream=None) -> LensDiffStatus:
        """Writes the normalised shifted raw PSF (S x S float32) to device `out`."""
        self._sync_custom(params)
        pp = abi.to_abi_params(params)
        st = abi.ld_status()
        self._lib.ld_raw_psf(self._h, ctypes.byref(pp), int(wavelength_index), _ptr(out), _stream(stream),
                             ctypes.byref(st))
        return LensDiffStatus(st)


def resolve_sizes(params: LensDiffParams) -> Tuple[int, int, int, int]:
    """(N_p, S, R_max, wavelength count) of the path for `params`."""
    L = abi.lib()
    pp = abi.to_abi_params(params)
    a, b, c, d = (ctypes.c_int32() for _ in range(4))
    L.ld_resolve_sizes(ctypes.byref(pp), ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(d))
    return a.value, b.value, c.value, d.value


def run_lensdiff_cuda(request: LensDiffRenderRequest, params: LensDiffParams,
                      cache: LensDiffPsfBankCache, error: Optional[list] = None) -> bool:
    """RunLensDiffCuda: True on success; on failure False and, if `error` is a
    list, the stage string appended to it (the `std::string* error` out-param)."""
    st = cache.render(request, params)
    if not st.ok and error is not None:
        error.append(st.stage)
    return st.ok


def image_request(src, dst, stream, src_origin=(0, 0), dst_origin=None, render_window=None,
                  frame_short_side: Optional[int] = None) -> LensDiffRenderRequest:
    """Request over two contiguous (H, W, 4) float32 device tensors."""
    h, w = int(src.shape[0]), int(src.shape[1])
    sx, sy = src_origin
    if dst_origin is None:
        dst_origin = src_origin
    dh, dw = int(dst.shape[0]), int(dst.shape[1])
    dx, dy = dst_origin
    sb = LensDiffImageRect(sx, sy, sx + w, sy + h)
    db = LensDiffImageRect(dx, dy, dx + dw, dy + dh)
    rw = db if render_window is None else LensDiffImageRect(*render_window)
    return LensDiffRenderRequest(
        renderWindow=rw,
        frameBounds=sb,
        src=LensDiffImageView(data=src, rowBytes=int(src.stride(0)) * 4, bounds=sb),
        dst=LensDiffImageView(data=dst, rowBytes=int(dst.stride(0)) * 4, bounds=db),
        frameShortSidePx=frame_short_side or min(w, h),
        hostEnabledCudaRender=True,
        cudaStream=stream,
    )
