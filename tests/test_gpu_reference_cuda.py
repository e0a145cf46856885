"""The reference's own CUDA chain, compiled unchanged (cuFFT transforms), as
the same-GPU comparator: it must reproduce the reference CPU renderer on a
small frame (so the timed comparator computes the path), and the library
must match it at the benchmark comparison's reference-expressible setting
(Spectral9, 3840x2160, pupil 512, kernel radius 512 px)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from lensdiff_b200 import synthetic as S  # noqa: E402
from lensdiff_b200.backend import LensDiffPsfBankCache, image_request  # noqa: E402
from lensdiff_b200.types import LensDiffApertureMode, LensDiffFftForm, LensDiffSpectralMode  # noqa: E402
from oracle import ref_lib as R  # noqa: E402
from tests.helpers import OUT_TOL, rel_err, with_matrices  # noqa: E402

pytestmark = pytest.mark.gpu


def _need():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not (R.cuda_available() and R.available()):
        pytest.skip("reference libraries not built")


def _ref_cuda(p, frame, instance=0):
    h, w = frame.shape[:2]
    src = torch.from_numpy(frame).cuda()
    dst = torch.full_like(src, -7.0)
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    R.cuda_render(p, src.data_ptr(), dst.data_ptr(), w, h, stream.cuda_stream, instance)
    stream.synchronize()
    return dst.cpu().numpy()


def _lens():
    p = S.base_params(120)
    p.apertureMode = LensDiffApertureMode.Polygon
    p.bladeCount = 7
    p.roundness = 0.2
    p.pupilResolution = 128
    p.phaseDefocus = 0.2
    p.maxKernelRadiusPx = S.radius_percent(20, 120)
    p.diffractionScalePx = 3.0
    p.spectralMode = LensDiffSpectralMode.Spectral5
    return p


def test_reference_cuda_chain_matches_reference_cpu():
    _need()
    p = _lens()
    frame = S.make_frame(200, 120, 14, 1.0, 60.0, seed=61)
    out = _ref_cuda(p, frame)
    ref = R.render(p, frame)
    assert rel_err(out, ref, ref[..., :3].max()) < OUT_TOL


def test_library_matches_reference_cuda_at_the_uhd_comparison_setting():
    _need()
    p, frame = S.workload_reference_uhd()
    out_ref = _ref_cuda(p, frame, instance=1)
    c = LensDiffPsfBankCache(0)
    try:
        stream = torch.cuda.Stream()
        src = torch.from_numpy(frame).cuda()
        dst = torch.full_like(src, -7.0)
        st = c.render(image_request(src, dst, stream, frame_short_side=p.frameShortSidePx),
                      with_matrices(p.copy(fftForm=LensDiffFftForm.OwnChosen)))
        stream.synchronize()
        assert st.ok, st
        out = dst.cpu().numpy()
    finally:
        c.close()
    assert rel_err(out, out_ref, out_ref[..., :3].max()) < OUT_TOL
