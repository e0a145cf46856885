"""Parity at the measured workloads' full sizes, against the FP64 oracle.

The three frame workloads the benchmark measures, at their full sizes:
  * small3: 1024x576, 64 highlights, pupil 256 -> PSF 512, 3 wavelengths;
  * hd16:   1920x1080, 512 highlights + 16 segments, 9 blades with rounding,
            obstruction and vanes, pupil 512 -> PSF 1024, Noll 2..15,
            16 wavelengths with Gaussian RGB responses;
  * uhd31:  3840x2160, 2048 highlights in [1, 1000], pupil 512 -> PSF 2048,
            31 wavelengths, chromatic focus (the headline workload).
Each is rendered in every transform form (the chosen form: tensor-core
BF16x3 PSF windows and FP16 frame spectra; the hand-written FP32 chain; the
cuFFT chain) and compared with one FP64 oracle render of the same inputs:
every bank kernel within 1e-4 of its peak, the output within 2e-4 of the
frame maximum.  The oracle is slow at UHD (tens of seconds on the host), so
each workload's oracle runs once per module.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from lensdiff_b200 import synthetic as S  # noqa: E402
from lensdiff_b200.backend import LensDiffPsfBankCache, image_request  # noqa: E402
from lensdiff_b200.types import LensDiffFftForm  # noqa: E402
from oracle import check as C  # noqa: E402
from tests.helpers import OUT_TOL, PSF_TOL  # noqa: E402

pytestmark = pytest.mark.gpu

WORKLOADS = {"small3": S.workload_small, "hd16": S.workload_hd, "uhd31": S.workload_uhd31}
FORMS = {"chosen": LensDiffFftForm.OwnChosen, "own_fp32": LensDiffFftForm.OwnFp32, "cufft": LensDiffFftForm.Cufft}

_ORACLE = {}


def _oracle(name):
    if name not in _ORACLE:
        p, frame = WORKLOADS[name]()
        _ORACLE[name] = (p, frame, C.OracleResult(p, frame))
    return _ORACLE[name]


@pytest.fixture(scope="module")
def cache():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    c = LensDiffPsfBankCache(0)
    yield c
    c.close()


def _render(cache, p, frame):
    stream = torch.cuda.Stream()
    src = torch.from_numpy(frame).cuda()
    dst = torch.full_like(src, -7.0)
    st = cache.render(image_request(src, dst, stream, frame_short_side=p.frameShortSidePx), p)
    assert st.ok, st
    stream.synchronize()
    assert cache.check_device_errors() == 0
    _, kernels, st2 = cache.export_psf_bank(p, stream)
    assert st2.ok, st2
    stream.synchronize()
    return dst.cpu().numpy(), kernels


@pytest.mark.parametrize("form", sorted(FORMS))
@pytest.mark.parametrize("name", ["small3", "hd16", "uhd31"])
def test_full_size_workload_error_vs_fp64_oracle(cache, name, form):
    p, frame, ref = _oracle(name)
    out, kernels = _render(cache, p.copy(fftForm=FORMS[form]), frame)
    rep = C.error_report(kernels, out, ref)
    print(f"{name} {form}: psf {rep['psf_vs_peak']:.2e} of peak, output {rep['out_vs_frame_max']:.2e} "
          f"of frame max (oracle {rep['oracle_seconds']} s)")
    assert rep["psf_vs_peak"] < PSF_TOL
    assert rep["out_vs_frame_max"] < OUT_TOL
    # the composite keeps the source's alpha and every pixel is written
    assert np.array_equal(out[..., 3], frame[..., 3])
