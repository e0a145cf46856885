"""Frame serving with continuous batching, over the library's ld_server_* C ABI.

A `LensDiffServer` keeps `slots` render slots on one GPU, each with its own
stream, device PSF-bank cache and worker thread.  `submit` queues a host RGBA
float32 frame and returns a ticket at once; frames start as soon as a slot is
free and the HBM budget admits them, so frames that arrive while others are
on the GPU overlap with them; frames with the same lens parameters go to the
slot that already holds their bank.  `wait` returns the frame's status and
latency (submit -> result on the host).
"""
from __future__ import annotations

import ctypes
from typing import Dict, Tuple

import numpy as np

from . import abi
from .backend import LensDiffStatus
from .types import LensDiffParams


class LensDiffServer:
    def __init__(self, device: int = 0, slots: int = 4, hbm_budget_bytes: int = 0):
        self._lib = abi.lib()
        self._h = ctypes.c_void_p()
        rc = self._lib.ld_server_create(ctypes.byref(self._h), device, slots, hbm_budget_bytes)
        if rc != abi.LD_OK:
            raise RuntimeError(f"ld_server_create failed ({rc})")
        self._frames: Dict[int, Tuple[np.ndarray, np.ndarray, abi.ld_params]] = {}

    def submit(self, src: np.ndarray, params: LensDiffParams, dst: np.ndarray = None) -> Tuple[int, np.ndarray]:
        """Queues one (H, W, 4) float32 frame (the whole frame is rendered; its
        short side sets the percent-based radii); returns (ticket, destination)."""
        src = np.ascontiguousarray(src, np.float32)
        h, w = src.shape[:2]
        if dst is None:
            dst = np.empty_like(src)
        pp = abi.to_abi_params(params.copy(frameShortSidePx=min(h, w)))
        t = ctypes.c_uint64()
        rc = self._lib.ld_server_submit(self._h, src.ctypes.data, dst.ctypes.data, w, h, ctypes.byref(pp),
                                        ctypes.byref(t))
        if rc != abi.LD_OK:
            raise RuntimeError(f"ld_server_submit failed ({rc})")
        self._frames[t.value] = (src, dst, pp)  # keep the buffers alive until wait
        return t.value, dst

    def wait(self, ticket: int, timeout_s: float = 60.0) -> Tuple[LensDiffStatus, float]:
        st = abi.ld_status()
        lat = ctypes.c_double()
        rc = self._lib.ld_server_wait(self._h, ticket, timeout_s, ctypes.byref(st), ctypes.byref(lat))
        if rc == abi.LD_ERR_TIMEOUT and st.code == 0:
            raise TimeoutError(f"frame {ticket} not done after {timeout_s} s")
        self._frames.pop(ticket, None)
        return LensDiffStatus(st), float(lat.value)

    def stats(self) -> dict:
        s = abi.ld_server_stats()
        self._lib.ld_server_get_stats(self._h, ctypes.byref(s))
        return {f: getattr(s, f) for f, _ in abi.ld_server_stats._fields_}

    def reset_stats(self) -> None:
        self._lib.ld_server_reset_stats(self._h)

    def close(self) -> None:
        if self._h:
            self._lib.ld_server_destroy(self._h)
            self._h = ctypes.c_void_p()
            self._frames.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
