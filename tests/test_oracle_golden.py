"""The FP64 oracle against the golden fixtures generated from the reference's
own CPU implementation (tests/golden/make_golden.py)."""
import json
import os

import numpy as np
import pytest

from oracle import ld_oracle as O
from tests.helpers import GOLDEN, OUT_TOL, PSF_TOL, golden_case, golden_cases, rel_err, spectrum_matrices

CASES = sorted(golden_cases().keys())


def test_first_zero_radii_match_reference():
    with open(os.path.join(GOLDEN, "first_zero.json")) as f:
        ref = json.load(f)
    for key, r0 in ref.items():
        n, s = (int(v) for v in key.split("x"))
        if s > 1024:
            continue  # the 2048 grids take a few seconds in numpy; covered on the GPU
        assert abs(O.reference_first_zero(n, s) - r0) < 1e-3, key


@pytest.mark.parametrize("name", CASES)
def test_bank_matches_reference(name):
    p, _, _, bank, wl, meta = golden_case(name)
    ob = O.build_psf_bank(p)
    assert [b.wavelength for b in ob.bins] == pytest.approx(wl)
    assert ob.support_radius == meta["support_radius"]
    for mine, ref in zip(ob.bins, bank):
        assert mine.full.shape == ref.shape
        assert rel_err(mine.full, ref, ref.max()) < PSF_TOL


@pytest.mark.parametrize("name", CASES)
def test_render_matches_reference(name):
    p, src, dst, _, _, _ = golden_case(name)
    bank = O.build_psf_bank(p)
    nat, sty = (None, None) if int(p.spectralMode) == 0 else spectrum_matrices(p)
    out = O.render(src, p, bank, nat, sty)
    assert rel_err(out, dst, dst[..., :3].max()) < OUT_TOL
    # the effect itself, against its own peak
    eff_ref = dst[..., :3] - src[..., :3]
    eff = out[..., :3] - src[..., :3]
    assert rel_err(eff, eff_ref, np.abs(eff_ref).max()) < 1e-3
