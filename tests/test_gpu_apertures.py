"""Custom aperture images and apodisation on the GPU, against the compiled
reference.

Custom: the host decodes the mask and hands the amplitudes to the library
(ld_set_custom_aperture, through the LensDiffParams.customApertureImage
extension); the reference's own loader gets the same decoded image through
its cache (ld_shim ldref_set_custom_aperture) and renders on the CPU.  Both
normalise / invert the image and sample it into the pupil, so renders and
raw PSFs must agree within the path's bars.  A new image must rebuild the
bank.  Apodisation: the Cosine and Gaussian pupil weights
(LensDiffCpuReference.cpp:670-680, applied at :751 and :817) with a polygon
and with a custom aperture.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from lensdiff_b200 import abi  # noqa: E402
from lensdiff_b200 import synthetic as S  # noqa: E402
from lensdiff_b200.backend import LensDiffPsfBankCache, image_request  # noqa: E402
from lensdiff_b200.types import (LensDiffApertureMode, LensDiffApodizationMode,  # noqa: E402
                                 LensDiffFftForm, LensDiffSpectralMode)
from oracle import ref_lib as R  # noqa: E402
from tests.helpers import OUT_TOL, PSF_TOL, rel_err, with_matrices  # noqa: E402
from tests.test_oracle_custom_aperture import custom_lens, mask_image  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cache():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not R.available():
        pytest.skip("compiled reference (oracle/_ref) not built")
    c = LensDiffPsfBankCache(0)
    yield c
    c.close()


def _render(cache, p, src):
    stream = torch.cuda.Stream()
    s = torch.from_numpy(np.ascontiguousarray(src, np.float32)).cuda()
    d = torch.full(src.shape, -7.0, device="cuda", dtype=torch.float32)
    st = cache.render(image_request(s, d, stream, frame_short_side=p.frameShortSidePx), p)
    torch.cuda.synchronize()
    assert cache.check_device_errors() == 0
    return st, d.cpu().numpy()


@pytest.mark.parametrize("norm,inv,apod,form", [
    (True, False, LensDiffApodizationMode.Flat, LensDiffFftForm.OwnFp32),
    (True, True, LensDiffApodizationMode.Cosine, LensDiffFftForm.OwnChosen),
    (False, False, LensDiffApodizationMode.Gaussian, LensDiffFftForm.OwnChosen),
])
def test_custom_aperture_render_matches_reference(cache, norm, inv, apod, form):
    img = mask_image()
    p = custom_lens(apodizationMode=apod, customApertureImage=img, customApertureNormalize=norm,
                    customApertureInvert=inv, spectralMode=LensDiffSpectralMode.Spectral5, phaseDefocus=0.15)
    R.set_custom_aperture(img, norm, inv)
    src = S.make_frame(200, 120, 14, 1.0, 60.0, seed=71)
    st, out = _render(cache, with_matrices(p.copy(fftForm=form)), src)
    assert st.ok, st
    ref = R.render(p, src)
    assert rel_err(out, ref, ref[..., :3].max()) < OUT_TOL


def test_custom_aperture_raw_psf_matches_reference(cache):
    img = mask_image(64, 40, seed=9)
    p = custom_lens(customApertureImage=img, spectralMode=LensDiffSpectralMode.Tristimulus)
    R.set_custom_aperture(img, True, False)
    _, S_, _ = R.sizes(p)
    out = torch.zeros(S_, S_, device="cuda")
    st = cache.raw_psf(p, 1, out, torch.cuda.current_stream())
    assert st.ok, st
    got = out.cpu().numpy().astype(np.float64)
    ref = R.raw_psf(p, 550.0).astype(np.float64)
    ref /= ref.sum()  # the reference's float normalising sum carries its own rounding
    assert rel_err(got, ref, ref.max()) < PSF_TOL


def test_new_custom_image_rebuilds_the_bank(cache):
    a, b = mask_image(seed=5), mask_image(seed=6)[:, ::-1].copy()
    src = S.make_frame(200, 120, 14, 1.0, 60.0, seed=72)
    outs = []
    for img in (a, b):
        p = custom_lens(customApertureImage=img, spectralMode=LensDiffSpectralMode.Tristimulus)
        st, out = _render(cache, with_matrices(p), src)
        assert st.ok and st.bank_rebuilt, st
        R.set_custom_aperture(img, True, False)
        ref = R.render(p, src)
        assert rel_err(out, ref, ref[..., :3].max()) < OUT_TOL
        outs.append(out)
    assert not np.array_equal(outs[0], outs[1])


def test_custom_mode_without_an_image_is_refused():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    c = LensDiffPsfBankCache(0)
    try:
        p = custom_lens(spectralMode=LensDiffSpectralMode.Tristimulus)
        st, _ = _render(c, with_matrices(p), S.make_frame(64, 48, 4, 1.0, 10.0, seed=73))
        assert st.code == abi.LD_ERR_ARG and st.stage == "custom-aperture-image-not-set"
    finally:
        c.close()


@pytest.mark.parametrize("apod", [LensDiffApodizationMode.Cosine, LensDiffApodizationMode.Gaussian])
@pytest.mark.parametrize("form", [LensDiffFftForm.OwnFp32, LensDiffFftForm.OwnChosen])
def test_apodised_polygon_matches_reference(cache, apod, form):
    p = S.base_params(144)
    p.apertureMode = LensDiffApertureMode.Polygon
    p.bladeCount = 7
    p.roundness = 0.3
    p.centralObstruction = 0.2
    p.pupilResolution = 128
    p.phaseDefocus = 0.2
    p.maxKernelRadiusPx = S.radius_percent(27, 144)
    p.diffractionScalePx = 3.0
    p.spectralMode = LensDiffSpectralMode.Spectral5
    p.apodizationMode = apod
    src = S.make_frame(224, 144, 20, 1.0, 80.0, seed=74)
    st, out = _render(cache, with_matrices(p.copy(fftForm=form)), src)
    assert st.ok, st
    ref = R.render(p, src)
    assert rel_err(out, ref, ref[..., :3].max()) < OUT_TOL
