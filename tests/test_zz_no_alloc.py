"""ld_raw_psf_noalloc: the raw-PSF entry point for callers that cannot
allocate device memory (a host application that owns and budgets all GPU
memory, a real-time thread that must not take cudaMalloc's implicit device
synchronisation).  Its scratch is a fixed file-scope device array, so the test
checks that two calls in a row both reproduce the allocating entry point
(ld_raw_psf) within the PSF tolerance, and that a request beyond the array's
limit is refused with an error instead of running.

This file sorts last so that a run stopping at the first failure has already
run every other test; it also passes alone in a fresh process.  The no-alloc
calls run before this test creates any library context, and one test runs
them in a fresh child process that never creates one, so the context-free
path (the first call's address lookup included) is exercised on its own.
"""
import ctypes
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from lensdiff_b200 import abi  # noqa: E402
from lensdiff_b200 import synthetic as S  # noqa: E402
from lensdiff_b200.backend import LensDiffPsfBankCache, resolve_sizes  # noqa: E402
from lensdiff_b200.types import LensDiffApertureMode, LensDiffSpectralMode  # noqa: E402
from tests.helpers import PSF_TOL, rel_err  # noqa: E402

pytestmark = pytest.mark.gpu


def _lens(pupil: int, radius_px: int, short_side: int = 288):
    p = S.base_params(short_side)
    p.apertureMode = LensDiffApertureMode.Polygon
    p.bladeCount = 7
    p.roundness = 0.3
    p.centralObstruction = 0.2
    p.vaneCount = 3
    p.vaneThickness = 0.03
    p.pupilResolution = pupil
    p.phaseDefocus = 0.3
    p.phaseComaX = 0.1
    p.chromaticFocus = 0.25
    p.maxKernelRadiusPx = S.radius_percent(radius_px, short_side)
    p.spectralMode = LensDiffSpectralMode.Tristimulus
    return p


def _noalloc(p, wl_index, out, stream):
    st = abi.ld_status()
    pp = abi.to_abi_params(p)
    rc = abi.lib().ld_raw_psf_noalloc(ctypes.byref(pp), wl_index, out.data_ptr(), stream.cuda_stream,
                                      ctypes.byref(st))
    return rc, st


def _reference_psf(p, wl_index, stream):
    """ld_raw_psf through a library context (the allocating entry point)."""
    _, S_, _, _ = resolve_sizes(p)
    cache = LensDiffPsfBankCache(0)
    ref = torch.zeros(S_, S_, device="cuda")
    st = cache.raw_psf(p, wl_index, ref, stream)
    assert st.ok, st
    stream.synchronize()
    ref_h = ref.cpu().numpy()
    cache.close()
    return ref_h


@pytest.mark.parametrize("pupil,radius,wl_index", [(256, 40, 0), (512, 200, 2)])
def test_noalloc_matches_allocating_entry_point_twice(pupil, radius, wl_index):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    p = _lens(pupil, radius)
    _, S_, _, _ = resolve_sizes(p)
    stream = torch.cuda.Stream()
    got = []
    for _ in range(2):  # before any library context exists in this test
        out = torch.full((S_, S_), -1.0, device="cuda")
        rc, st = _noalloc(p, wl_index, out, stream)
        assert rc == abi.LD_OK, st.stage
        stream.synchronize()
        got.append(out.cpu().numpy())
    ref_h = _reference_psf(p, wl_index, stream)
    for g in got:
        assert rel_err(g, ref_h, ref_h.max()) < PSF_TOL
        assert abs(float(g.sum()) - 1.0) < 1e-5


_CHILD = r"""
import ctypes, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
from lensdiff_b200 import abi
from tests.test_zz_no_alloc import _lens, _noalloc
from lensdiff_b200.backend import resolve_sizes
p = _lens(256, 40)
_, S_, _, _ = resolve_sizes(p)
stream = torch.cuda.Stream()
outs = []
for _ in range(2):
    out = torch.full((S_, S_), -1.0, device="cuda")
    rc, st = _noalloc(p, 1, out, stream)
    assert rc == abi.LD_OK, st.stage
    stream.synchronize()
    outs.append(out.cpu().numpy())
np.save(sys.argv[2], np.stack(outs))
"""


def test_noalloc_in_a_fresh_process_without_any_context():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "psf.npy")
        res = subprocess.run([sys.executable, "-c", _CHILD, root, path], capture_output=True, text=True,
                             timeout=300)
        assert res.returncode == 0, res.stderr[-2000:]
        got = np.load(path)
    p = _lens(256, 40)
    ref_h = _reference_psf(p, 1, torch.cuda.Stream())
    for g in got:
        assert rel_err(g, ref_h, ref_h.max()) < PSF_TOL


def test_noalloc_rejects_sizes_beyond_its_scratch():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    p = _lens(1024, 200)  # pupil 1024 -> PSF grid 2048, above the limit
    out = torch.zeros(16, device="cuda")
    rc, st = _noalloc(p, 0, out, torch.cuda.Stream())
    assert rc == abi.LD_ERR_ARG
    assert b"exceeds-no-alloc" in st.stage
    assert np.all(out.cpu().numpy() == 0.0)
