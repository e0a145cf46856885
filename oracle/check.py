"""Error of a CUDA-path result against the FP64 oracle — TEST INFRASTRUCTURE.

Used as the checker by tests/ and by bench.py (outside its timed regions) to
state each result's error in the path's two measures:

  * PSF: max |kernel - oracle kernel| / oracle kernel peak, over every bank
    kernel (the normalised, cropped and tapered kernels of
    populatePsfBankCacheFromBaseKernels, LensDiffCpuReference.cpp:1616-1656);
  * output: max |output - oracle output| / oracle frame maximum (linear RGB
    of RunLensDiffCpuReference's composite, LensDiffCpuReference.cpp:2073-2261).

The oracle is the FP64 restatement in oracle/ld_oracle.py, itself pinned to
the reference's compiled CPU code by the golden fixtures.
"""
from __future__ import annotations

import time
from typing import Dict, Optional, Sequence

import numpy as np

from . import ld_oracle as O

ORACLE_NAME = "FP64 numpy restatement of the reference CPU path (oracle/ld_oracle.py)"


def oracle_matrices(p):
    """The (natural, style) spectral matrices the render uses."""
    if int(p.spectralMode) == 0:
        return None, None
    if int(getattr(p, "rgbMode", 0)) == 1:  # Gaussian responses
        m = O.gaussian_rgb_matrix(O.wavelengths(p), p.rgbGaussCenterNm, p.rgbGaussSigmaNm)
        return m, m
    return np.array(p.naturalMatrix, np.float64), np.array(p.styleMatrix, np.float64)


class OracleResult:
    """FP64 bank and render of one (params, frame) pair, computed once."""

    def __init__(self, p, frame: np.ndarray):
        t = time.perf_counter()
        self.bank = O.build_psf_bank(p)
        nat, sty = oracle_matrices(p)
        self.out = O.render(frame, p, self.bank, nat, sty)
        self.seconds = time.perf_counter() - t
        self.frame_max = float(self.out[..., :3].max())


def psf_error(kernels: Sequence[np.ndarray], ref: OracleResult) -> float:
    """Largest error of any bank kernel, relative to that kernel's oracle peak."""
    bins = ref.bank.bins
    if len(kernels) != len(bins):
        raise ValueError(f"{len(kernels)} kernels against {len(bins)} oracle bins")
    worst = 0.0
    for k, b in zip(kernels, bins):
        r = b.full
        if k.shape != r.shape:
            raise ValueError(f"kernel shape {k.shape} against oracle {r.shape}")
        worst = max(worst, float(np.abs(np.asarray(k, np.float64) - r).max() / max(float(r.max()), 1e-30)))
    return worst


def output_error(out: np.ndarray, ref: OracleResult) -> float:
    """max |out - oracle| over every channel, relative to the oracle's RGB maximum."""
    return float(np.abs(np.asarray(out, np.float64) - ref.out).max() / max(ref.frame_max, 1e-30))


def error_report(kernels: Optional[Sequence[np.ndarray]], out: np.ndarray, ref: OracleResult) -> Dict:
    return {
        "psf_vs_peak": psf_error(kernels, ref) if kernels is not None else None,
        "out_vs_frame_max": output_error(out, ref),
        "bars": {"psf_vs_peak": 1e-4, "out_vs_frame_max": 2e-4},
        "oracle": ORACLE_NAME,
        "oracle_seconds": round(ref.seconds, 1),
    }
