"""The Custom aperture mode's restatement pinned to the reference's own code
(no GPU).  The reference decodes the mask file with WIC / ImageIO, absent
here, so the checker seeds the reference loader's own cache with an image
decoded in the test (ref_shim.cpp ldref_set_custom_aperture); the
reference's normalise / invert (LensDiffApertureImage.cpp:367-399) and its
sampling into the pupil (LensDiffCpuReference.cpp:707-756) then run
unchanged and the oracle (oracle/ld_oracle.py custom_pupil_amplitude) must
agree with them."""
import numpy as np
import pytest

from lensdiff_b200 import synthetic as S
from lensdiff_b200.types import LensDiffApertureMode, LensDiffApodizationMode
from oracle import ld_oracle as O
from oracle import ref_lib as R


def mask_image(h=48, w=80, seed=5):
    """An elliptical opening with a bar, on noise, in arbitrary units."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    img = np.zeros((h, w), np.float32)
    img[((xx - w / 2) ** 2 / (0.38 * w) ** 2 + (yy - h / 2) ** 2 / (0.38 * h) ** 2) < 1] = 200.0
    img[int(0.42 * h):int(0.58 * h), :] = 30.0
    return img + rng.uniform(0, 10, img.shape).astype(np.float32)


def custom_lens(**kw):
    p = S.base_params(120)
    p.apertureMode = LensDiffApertureMode.Custom
    p.pupilResolution = 128
    p.rotationDeg = 17.0
    p.pupilDecenterX = 0.03
    p.maxKernelRadiusPx = S.radius_percent(20, 120)
    p.diffractionScalePx = 3.0
    for k, v in kw.items():
        setattr(p, k, v)
    return p


@pytest.fixture(scope="module", autouse=True)
def need_reference():
    if not R.available():
        pytest.skip("compiled reference (oracle/_ref) not built")


@pytest.mark.parametrize("norm,inv,apod,shape", [
    (True, False, LensDiffApodizationMode.Flat, (48, 80)),
    (True, True, LensDiffApodizationMode.Cosine, (48, 80)),
    (False, False, LensDiffApodizationMode.Gaussian, (80, 48)),
])
def test_custom_pupil_matches_reference(norm, inv, apod, shape):
    img = mask_image(*shape)
    p = custom_lens(apodizationMode=apod, customApertureImage=img, customApertureNormalize=norm,
                    customApertureInvert=inv)
    R.set_custom_aperture(img, norm, inv)
    ref, _ = R.pupil(p)
    got = O.pupil_amplitude(p)
    assert (ref > 0).sum() > 1000
    assert np.abs(got - ref).max() <= 2e-7 * max(1.0, float(ref.max()))


def test_custom_raw_psf_matches_reference():
    img = mask_image()
    p = custom_lens(customApertureImage=img)
    R.set_custom_aperture(img, True, False)
    ref = R.raw_psf(p, 550.0).astype(np.float64)
    amp = O.pupil_amplitude(p)
    got = O.raw_psf(amp, None, ref.shape[0])
    ref = ref / ref.sum()
    assert np.abs(got - ref).max() / ref.max() < 1e-5
