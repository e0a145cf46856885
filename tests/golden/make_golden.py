"""Generates the golden fixtures in this folder from the reference's own CPU
implementation (oracle/_ref/libldref.so, built from the reference sources by
oracle/Makefile).  Run from the repository root:

    python tests/golden/make_golden.py

The reference ships no golden outputs of its own; these fixtures pin the FP64
oracle (oracle/ld_oracle.py) to the reference on machines where the
reference sources are not present.
"""
from __future__ import annotations

import json
import os
import sys
import zlib

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from lensdiff_b200 import synthetic as S  # noqa: E402
from lensdiff_b200.types import (  # noqa: E402
    LensDiffApertureMode,
    LensDiffEnergyMode,
    LensDiffLookMode,
    LensDiffSpectralMode,
    LensDiffSpectrumStyle,
)
from oracle import ld_oracle as O  # noqa: E402
from oracle import ref_lib as R  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def golden_params():
    """Small lens settings the golden renders use (frames 128x72 / 97x61)."""
    base = S.base_params(72)
    base.apertureMode = LensDiffApertureMode.Polygon
    base.bladeCount = 7
    base.roundness = 0.25
    base.rotationDeg = 12.0
    base.centralObstruction = 0.2
    base.vaneCount = 3
    base.vaneThickness = 0.03
    base.pupilResolution = 64
    base.phaseDefocus = 0.3
    base.phaseComaX = 0.1
    base.phaseSpherical = -0.15
    base.maxKernelRadiusPx = S.radius_percent(14, 72)
    base.diffractionScalePx = 2.0
    cases = {}
    cases["tristimulus_physical_augment"] = base.copy(spectralMode=LensDiffSpectralMode.Tristimulus)
    cases["mono_physical_augment"] = base.copy(spectralMode=LensDiffSpectralMode.Mono,
                                               apertureMode=LensDiffApertureMode.Circle)
    cases["spectral9_chromatic"] = base.copy(spectralMode=LensDiffSpectralMode.Spectral9, chromaticFocus=0.3,
                                             chromaticSpread=0.2, diffractionScalePx=0.4)
    cases["spectral5_split_preserve"] = base.copy(spectralMode=LensDiffSpectralMode.Spectral5,
                                                  lookMode=LensDiffLookMode.Split,
                                                  energyMode=LensDiffEnergyMode.Preserve, corePreserve=0.1,
                                                  coreShoulder=0.4, structureGain=1.5)
    cases["tristimulus_style_force"] = base.copy(spectralMode=LensDiffSpectralMode.Tristimulus,
                                                 spectrumStyle=LensDiffSpectrumStyle.CyanMagenta,
                                                 spectrumForce=0.6, spectrumSaturation=1.3)
    # after the effect: scatter, creative fringe, the resolution-aware working
    # frame (percentages of the 2160-pixel optics short side when
    # resolution-aware; 4320 halves the working frame, 1080 doubles it)
    cases["tristimulus_scatter_fringe"] = base.copy(spectralMode=LensDiffSpectralMode.Tristimulus,
                                                    scatterAmount=0.6, scatterRadius=8.0, creativeFringe=2.5)
    aware = base.copy(resolutionAware=True, diffractionScalePx=2.0 * 72 / 2160)
    cases["spectral5_aware_up_scatter_preserve"] = aware.copy(
        spectralMode=LensDiffSpectralMode.Spectral5, frameShortSidePx=1080,
        maxKernelRadiusPx=S.radius_percent(20, 2160), energyMode=LensDiffEnergyMode.Preserve, corePreserve=0.1,
        scatterAmount=0.4, scatterRadius=0.4, creativeFringe=0.05)
    cases["mono_aware_down_fringe"] = aware.copy(
        spectralMode=LensDiffSpectralMode.Mono, apertureMode=LensDiffApertureMode.Circle, frameShortSidePx=4320,
        maxKernelRadiusPx=S.radius_percent(10, 2160), creativeFringe=0.1)
    # DaVinci Intermediate source and output encoding (frames of encoded values)
    cases["spectral5_davinci_transfer"] = base.copy(spectralMode=LensDiffSpectralMode.Spectral5, inputTransfer=1)
    return cases


def params_json(p) -> dict:
    d = {}
    for k, v in vars(p).items():
        if v is None or isinstance(v, (str,)):
            d[k] = v
        elif isinstance(v, (list, tuple)):
            d[k] = [float(x) for x in v]
        else:
            d[k] = float(v) if isinstance(v, float) else int(v)
    return d


def main() -> None:
    if not R.build():
        raise SystemExit("reference sources not available")
    # spectrum matrices of every reference mode and style
    mats = {}
    for mode in (LensDiffSpectralMode.Tristimulus, LensDiffSpectralMode.Spectral5, LensDiffSpectralMode.Spectral9):
        for style in LensDiffSpectrumStyle:
            p = S.base_params(1080).copy(spectralMode=mode, spectrumStyle=style)
            wl = O.MODE_WAVELENGTHS[int(mode)]
            nat, sty, cnt = R.spectrum_matrices(p, wl)
            mats[f"{mode.name}/{style.name}"] = {"wavelengths": wl, "natural": nat.tolist(),
                                                 "style": sty.tolist(), "binCount": cnt}
    with open(os.path.join(OUT, "spectrum_matrices.json"), "w") as f:
        json.dump(mats, f, indent=1)
    # first-minimum calibration radii
    r0 = {f"{n}x{s}": R.first_zero(n, s) for n, s in
          [(64, 512), (128, 512), (256, 512), (256, 1024), (512, 1024), (512, 2048), (1024, 2048)]}
    with open(os.path.join(OUT, "first_zero.json"), "w") as f:
        json.dump(r0, f, indent=1)
    # renders and banks
    cases = golden_params()
    meta = {}
    for name, p in cases.items():
        w, h = (128, 72) if "spectral9" not in name else (97, 61)
        lo, hi = (0.55, 0.8) if "davinci" in name else (1.0, 80.0)  # encoded values decode to about 1-40
        frame = S.make_frame(w, h, 12, lo, hi, seed=zlib.crc32(name.encode()) % 1000 + 11)
        out = R.render(p, frame)
        wl, fulls, _, _, sup = R.bank(p)
        np.savez_compressed(os.path.join(OUT, f"render_{name}.npz"), src=frame, dst=out)
        np.savez_compressed(os.path.join(OUT, f"bank_{name}.npz"),
                            **{f"full_{i}": k for i, k in enumerate(fulls)}, wavelengths=np.array(wl))
        meta[name] = {"params": params_json(p), "support_radius": sup, "size": [w, h]}
    with open(os.path.join(OUT, "cases.json"), "w") as f:
        json.dump(meta, f, indent=1)
    print("golden fixtures written to", OUT)


if __name__ == "__main__":
    main()
