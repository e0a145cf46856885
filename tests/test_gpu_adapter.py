"""The drop-in boundary end to end: the plugin's own call
RunLensDiffCuda(const LensDiffRenderRequest&, const LensDiffParams&,
LensDiffPsfBankCache&, std::string*) (LensDiffCuda.h:7-10) as implemented by
lensdiff_b200/adapter/LensDiffCudaB200.cpp, compiled against the reference's
headers and spectrum code (oracle/_ref/libldadapter.so, oracle/Makefile),
driven with the reference's request and parameter types, against the
reference's CPU renderer on the same inputs.
"""
import ctypes
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from lensdiff_b200 import abi  # noqa: E402
from lensdiff_b200 import synthetic as S  # noqa: E402
from lensdiff_b200.types import (LensDiffApertureMode, LensDiffEnergyMode, LensDiffPhaseMode,  # noqa: E402
                                 LensDiffSpectralMode)
from oracle import ref_lib as R  # noqa: E402
from tests.helpers import OUT_TOL, rel_err  # noqa: E402

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
ADAPTER = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libldadapter.so")


@pytest.fixture(scope="module")
def adapter():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not (os.path.exists(ADAPTER) and R.available()):
        pytest.skip("adapter harness / compiled reference not built")
    return _adapter_lib()


def _adapter_lib():
    abi.lib()  # the adapter resolves the library's symbols
    L = ctypes.CDLL(ADAPTER)
    i, ll, vp = ctypes.c_int, ctypes.c_longlong, ctypes.c_void_p
    L.ldadapter_render.argtypes = [ctypes.POINTER(abi.ld_params), vp, i, i, i, i, ll, vp, i, i, i, i, ll,
                                   i, i, i, i, vp, i, ctypes.c_char_p, i]
    L.ldadapter_render.restype = i
    return L


def _run(L, p, src, stream, host_enabled=1, null_src=False, window=None):
    h, w = src.shape[:2]
    s = torch.from_numpy(np.ascontiguousarray(src, np.float32)).cuda()
    d = torch.full_like(s, -7.0)
    pp = abi.to_abi_params(p)
    err = ctypes.create_string_buffer(256)
    rx1, ry1, rx2, ry2 = window or (0, 0, w, h)
    ok = L.ldadapter_render(ctypes.byref(pp), None if null_src else s.data_ptr(), 0, 0, w, h, w * 16,
                            d.data_ptr(), 0, 0, w, h, w * 16, rx1, ry1, rx2, ry2,
                            stream.cuda_stream if stream is not None else None, host_enabled, err, 256)
    torch.cuda.synchronize()
    return ok, err.value.decode(), d.cpu().numpy()


def _lens(**kw):
    p = S.base_params(120)
    p.apertureMode = LensDiffApertureMode.Polygon
    p.bladeCount = 8
    p.roundness = 0.25
    p.pupilResolution = 128
    p.phaseDefocus = 0.2
    p.maxKernelRadiusPx = S.radius_percent(22, 120)
    p.diffractionScalePx = 3.0
    p.spectralMode = LensDiffSpectralMode.Spectral5
    for k, v in kw.items():
        setattr(p, k, v)
    return p


@pytest.mark.parametrize("kw", [{}, {"spectralMode": LensDiffSpectralMode.Mono},
                                {"energyMode": LensDiffEnergyMode.Preserve, "effectGain": 0.7},
                                {"phaseMode": LensDiffPhaseMode.Enabled, "phaseFieldStrength": 1.0,
                                 "phaseFieldComaRadial": 0.3, "phaseFieldDefocus": 0.1},
                                {"scatterAmount": 0.5, "scatterRadius": 8.0, "creativeFringe": 1.5},
                                {"resolutionAware": True, "frameShortSidePx": 1080,
                                 "maxKernelRadiusPx": 1.25, "diffractionScalePx": 0.2}])
def test_run_lensdiff_cuda_matches_reference_cpu(adapter, kw):
    p = _lens(**kw)
    src = S.make_frame(200, 120, 14, 1.0, 60.0, seed=41)
    ok, err, out = _run(adapter, p, src, torch.cuda.Stream())
    assert ok == 1, err
    ref = R.render(p, src)
    assert rel_err(out, ref, ref[..., :3].max()) < OUT_TOL


def test_run_lensdiff_cuda_error_strings(adapter):
    p = _lens()
    src = S.make_frame(64, 48, 4, 1.0, 10.0, seed=42)
    ok, err, _ = _run(adapter, p, src, torch.cuda.Stream(), host_enabled=0)
    assert ok == 0 and err == "cuda-render-not-enabled-by-host"  # LensDiffCuda.cu:4646-4651
    ok, err, _ = _run(adapter, p, src, None)
    assert ok == 0 and err == "cuda-render-not-enabled-by-host"
    ok, err, _ = _run(adapter, p, src, torch.cuda.Stream(), null_src=True)
    assert ok == 0 and err == "missing-source-or-destination-cuda-buffer"  # :4652-4657


_CHILD = r"""
import sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
from tests.test_gpu_adapter import _adapter_lib, _lens, _run
from lensdiff_b200 import synthetic as S
L = _adapter_lib()
p = _lens()
src = S.make_frame(200, 120, 14, 1.0, 60.0, seed=41)
ok, err, out = _run(L, p, src, torch.cuda.Stream())
assert ok == 1, err
np.save(sys.argv[2], out)
"""


@pytest.mark.parametrize("form", ["chosen", "fp32", "cufft"])
def test_run_lensdiff_cuda_form_switch(adapter, form):
    """LENSDIFF_B200_FFT_FORM selects the transform chain behind the plugin's
    call (read once per process, so each form runs in its own process)."""
    import subprocess
    import sys
    import tempfile

    root = os.path.dirname(HERE)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "out.npy")
        env = dict(os.environ, LENSDIFF_B200_FFT_FORM=form, LENSDIFF_B200_HBM_BUDGET_MB="4096")
        res = subprocess.run([sys.executable, "-c", _CHILD, root, path], capture_output=True, text=True,
                             timeout=600, env=env)
        assert res.returncode == 0, res.stderr[-2000:]
        out = np.load(path)
    p = _lens()
    ref = R.render(p, S.make_frame(200, 120, 14, 1.0, 60.0, seed=41))
    assert rel_err(out, ref, ref[..., :3].max()) < OUT_TOL
