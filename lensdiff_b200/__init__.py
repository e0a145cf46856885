"""lensdiff_b200 — B200-native (sm_100a) LensDiff diffraction path.

The device path lives in liblensdiff_b200.so (csrc/, C ABI in
include/lensdiff_b200.h); this package mirrors the reference's request and
parameter types and its CUDA backend entry point for Python callers.
"""
from .types import *  # noqa: F401,F403
from .types import (
    LensDiffImageRect,
    LensDiffImageView,
    LensDiffParams,
    LensDiffRenderRequest,
    resolved_wavelengths,
)

__all__ = [
    "LensDiffImageRect",
    "LensDiffImageView",
    "LensDiffParams",
    "LensDiffRenderRequest",
    "resolved_wavelengths",
    "LensDiffPsfBankCache",
    "run_lensdiff_cuda",
    "image_request",
    "resolve_sizes",
]


def __getattr__(name):
    # the native entry points load liblensdiff_b200.so on first use
    if name in ("LensDiffPsfBankCache", "run_lensdiff_cuda", "image_request", "resolve_sizes",
                "LensDiffStatus"):
        from . import backend
        return getattr(backend, name)
    raise AttributeError(name)
