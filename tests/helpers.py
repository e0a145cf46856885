"""Shared test helpers: golden fixtures, parameter decoding, tolerances."""
from __future__ import annotations

import json
import os

import numpy as np

from lensdiff_b200.types import LensDiffParams, LensDiffSpectrumStyle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# Parity bars of the path: normalised PSF within 1e-4 of its peak, output
# linear RGB within 2e-4 of the frame maximum.
PSF_TOL = 1e-4
OUT_TOL = 2e-4

_ENUM_FIELDS = {f: type(getattr(LensDiffParams(), f)) for f in vars(LensDiffParams())
                if hasattr(type(getattr(LensDiffParams(), f)), "__members__")}


def params_from_json(d: dict) -> LensDiffParams:
    p = LensDiffParams()
    for k, v in d.items():
        if k in _ENUM_FIELDS:
            setattr(p, k, _ENUM_FIELDS[k](int(v)))
        elif isinstance(getattr(p, k), bool):
            setattr(p, k, bool(v))
        elif isinstance(getattr(p, k), int) and not isinstance(getattr(p, k), bool):
            setattr(p, k, int(v))
        else:
            setattr(p, k, v if not isinstance(v, list) else list(v))
    return p


def golden_cases():
    with open(os.path.join(GOLDEN, "cases.json")) as f:
        return json.load(f)


def golden_case(name: str):
    meta = golden_cases()[name]
    p = params_from_json(meta["params"])
    r = np.load(os.path.join(GOLDEN, f"render_{name}.npz"))
    b = np.load(os.path.join(GOLDEN, f"bank_{name}.npz"))
    n = sum(1 for k in b.files if k.startswith("full_"))
    bank = [b[f"full_{i}"] for i in range(n)]
    return p, r["src"], r["dst"], bank, [float(x) for x in b["wavelengths"]], meta


def spectrum_matrices(p: LensDiffParams):
    """(natural, style) 3 x B matrices of a reference spectral mode from the
    golden fixture of BuildLensDiffSpectrumConfig."""
    with open(os.path.join(GOLDEN, "spectrum_matrices.json")) as f:
        mats = json.load(f)
    key = f"{p.spectralMode.name}/{LensDiffSpectrumStyle(p.spectrumStyle).name}"
    m = mats[key]
    return np.array(m["natural"], np.float64), np.array(m["style"], np.float64)


def with_matrices(p: LensDiffParams) -> LensDiffParams:
    """Copy of a reference-mode parameter set carrying its spectral matrices
    (the plugin passes them in from its own BuildLensDiffSpectrumConfig)."""
    if int(p.spectralMode) == 0:
        return p.copy()
    nat, sty = spectrum_matrices(p)
    return p.copy(naturalMatrix=nat.tolist(), styleMatrix=sty.tolist())


def rel_err(a: np.ndarray, b: np.ndarray, scale: float) -> float:
    return float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max() / max(scale, 1e-30))
