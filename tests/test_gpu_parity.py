"""CUDA path vs the FP64 oracle, through the C ABI (liblensdiff_b200.so).

Tolerances: normalised PSF within 1e-4 of its peak; output linear RGB within
2e-4 of the frame maximum (tests/helpers.py).  The oracle itself is pinned to
the reference's CPU code by tests/test_oracle_golden.py.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from lensdiff_b200 import synthetic as S  # noqa: E402
from lensdiff_b200.backend import LensDiffPsfBankCache, image_request, resolve_sizes, run_lensdiff_cuda  # noqa: E402
from lensdiff_b200.types import (  # noqa: E402
    LensDiffApertureMode,
    LensDiffFftForm,
    LensDiffLookMode,
    LensDiffRgbMode,
    LensDiffSpectralMode,
    LensDiffSpectrumStyle,
)
from oracle import ld_oracle as O  # noqa: E402
from tests.helpers import OUT_TOL, PSF_TOL, golden_case, golden_cases, rel_err, spectrum_matrices, with_matrices  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cache():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    c = LensDiffPsfBankCache(0)
    yield c
    c.close()


def _oracle_matrices(p):
    if int(p.spectralMode) == 0:
        return None, None
    if p.rgbMode == LensDiffRgbMode.Gaussian:
        m = O.gaussian_rgb_matrix(O.wavelengths(p), p.rgbGaussCenterNm, p.rgbGaussSigmaNm)
        return m, m
    return np.array(p.naturalMatrix, np.float64), np.array(p.styleMatrix, np.float64)


_STREAM = []


def side_stream():
    """A non-default stream: like the plugin host, the path requires a real
    cudaStream (handle 0 is rejected as at LensDiffCuda.cu:4646-4651)."""
    if not _STREAM:
        _STREAM.append(torch.cuda.Stream())
    return _STREAM[0]


def render_gpu(cache, p, src, src_origin=(0, 0), dst_shape=None, dst_origin=None, render_window=None):
    stream = side_stream()
    s = torch.from_numpy(np.ascontiguousarray(src, np.float32)).cuda()
    if dst_shape is None:
        dst_shape = src.shape
    d = torch.full(dst_shape, -7.0, device="cuda", dtype=torch.float32)
    req = image_request(s, d, stream, src_origin=src_origin, dst_origin=dst_origin,
                        render_window=render_window, frame_short_side=p.frameShortSidePx)
    st = cache.render(req, p)
    torch.cuda.synchronize()
    assert cache.check_device_errors() == 0, "a kernel recorded a device error (timeout or bad bulk copy)"
    return d.cpu().numpy(), st


def small_lens(**kw):
    p = S.base_params(144)
    p.apertureMode = LensDiffApertureMode.Polygon
    p.bladeCount = 6
    p.roundness = 0.2
    p.pupilResolution = 128
    p.phaseDefocus = 0.25
    p.phaseSpherical = 0.1
    p.maxKernelRadiusPx = S.radius_percent(29, 144)
    p.diffractionScalePx = 3.0
    p.spectralMode = LensDiffSpectralMode.Tristimulus
    for k, v in kw.items():
        setattr(p, k, v)
    return p


# ---------------------------------------------------------------- PSF ------
@pytest.mark.parametrize("wl_index", [0, 2])
def test_raw_psf_matches_oracle(cache, wl_index):
    p = small_lens(chromaticFocus=0.4, centralObstruction=0.25, vaneCount=3, vaneThickness=0.04, rotationDeg=17.0)
    np_, S_, R, B = resolve_sizes(p)
    out = torch.zeros(S_, S_, device="cuda")
    st = cache.raw_psf(p, wl_index, out, torch.cuda.current_stream())
    assert st.ok, st
    torch.cuda.synchronize()
    wl = O.wavelengths(p)[wl_index]
    coeffs, en, _ = O.wavelength_phase_setup(p, wl)
    ref = O.raw_psf(O.pupil_amplitude(p), O.phase_waves(p, coeffs, en), S_)
    got = out.cpu().numpy()
    assert abs(got.sum() - 1.0) < 1e-5
    assert rel_err(got, ref, ref.max()) < PSF_TOL


@pytest.mark.parametrize("name", sorted(golden_cases().keys()))
def test_bank_matches_reference_fixture(cache, name):
    p, _, _, bank, wl, meta = golden_case(name)
    if p.lookMode != LensDiffLookMode.Physical:
        p = p.copy(lookMode=LensDiffLookMode.Physical, energyMode=1)
    wls, kernels, st = cache.export_psf_bank(p, torch.cuda.current_stream())
    assert st.ok, st
    assert st.support_radius == meta["support_radius"]
    assert wls == pytest.approx(wl)
    for k, ref in zip(kernels, bank):
        assert k.shape == ref.shape
        assert rel_err(k, ref, ref.max()) < PSF_TOL


def test_bank_tier_x_matches_oracle(cache):
    p, _ = S.workload_hd()
    p = S.scaled_down(p, 144, pupil=128, max_radius_px=24)
    p.wavelengthsNm = list(np.linspace(400.0, 700.0, 16))
    wls, kernels, st = cache.export_psf_bank(p, torch.cuda.current_stream())
    assert st.ok, st
    ob = O.build_psf_bank(p)
    assert len(kernels) == 16
    for k, b in zip(kernels, ob.bins):
        assert k.shape == b.full.shape
        assert rel_err(k, b.full, b.full.max()) < PSF_TOL


# ------------------------------------------------------------- render ------
@pytest.mark.parametrize("name", sorted(golden_cases().keys()))
def test_render_matches_reference_fixture(cache, name):
    p, src, dst, _, _, _ = golden_case(name)
    p = with_matrices(p)
    out, st = render_gpu(cache, p, src)
    torch.cuda.synchronize()
    assert st.ok, st
    assert rel_err(out, dst, dst[..., :3].max()) < OUT_TOL
    eff_ref = dst[..., :3] - src[..., :3]
    assert rel_err(out[..., :3] - src[..., :3], eff_ref, np.abs(eff_ref).max()) < 2e-3


@pytest.mark.parametrize("mode", [LensDiffSpectralMode.Mono, LensDiffSpectralMode.Tristimulus,
                                  LensDiffSpectralMode.Spectral5, LensDiffSpectralMode.Spectral9])
def test_render_modes_match_oracle(cache, mode):
    p = with_matrices(small_lens(spectralMode=mode))
    src = S.make_frame(256, 144, 24, 1.0, 100.0, seed=5)
    out, st = render_gpu(cache, p, src)
    assert st.ok, st
    bank = O.build_psf_bank(p)
    nat, sty = _oracle_matrices(p)
    ref = O.render(src, p, bank, nat, sty)
    assert rel_err(out, ref, ref[..., :3].max()) < OUT_TOL


def test_render_tier_x_hd_lens_matches_oracle(cache):
    p, _ = S.workload_hd()
    p = S.scaled_down(p, 120, pupil=128, max_radius_px=20)
    src = S.make_frame(200, 120, 40, 1.0, 100.0, seed=9, segments=4)
    out, st = render_gpu(cache, p, src)
    assert st.ok, st
    ref = O.render(src, p, O.build_psf_bank(p), *_oracle_matrices(p))
    assert rel_err(out, ref, ref[..., :3].max()) < OUT_TOL


@pytest.mark.parametrize("form", [LensDiffFftForm.OwnFp32, LensDiffFftForm.OwnChosen])
def test_render_window_origin_and_odd_sizes(cache, form):
    """Odd frame sizes and shifted origins; in the chosen form the row
    spectra rows are padded to a multiple of 4 (117 -> 120) and their
    exponent bytes to a multiple of 16 for the column pass's bulk copy."""
    p = with_matrices(small_lens(fftForm=form))
    src = S.make_frame(203, 117, 20, 1.0, 60.0, seed=3)
    origin = (40, -13)
    dst_origin = (30, -20)
    dst_shape = (140, 230, 4)
    window = (45, -10, 220, 100)
    out, st = render_gpu(cache, p, src, src_origin=origin, dst_shape=dst_shape, dst_origin=dst_origin,
                         render_window=window)
    assert st.ok, st
    ref = O.render(src, p, O.build_psf_bank(p), *_oracle_matrices(p), src_origin=origin,
                   dst_bounds=(dst_origin[0], dst_origin[1], dst_origin[0] + dst_shape[1],
                               dst_origin[1] + dst_shape[0]),
                   render_window=window)
    inside = np.zeros(dst_shape[:2], bool)
    x1, y1 = window[0] - dst_origin[0], window[1] - dst_origin[1]
    x2, y2 = window[2] - dst_origin[0], window[3] - dst_origin[1]
    inside[max(0, y1):y2, max(0, x1):x2] = True
    assert np.all(out[~inside] == -7.0)  # untouched outside the render window
    assert rel_err(out[inside], ref[inside], ref[inside][..., :3].max()) < OUT_TOL


def test_luma_lock_and_saturation(cache):
    p = with_matrices(small_lens(spectrumStyle=LensDiffSpectrumStyle.WarmCool, spectrumForce=0.7,
                                 spectrumSaturation=1.4))
    nat, sty = spectrum_matrices(p)
    src = S.make_frame(160, 96, 16, 1.0, 100.0, seed=4)
    out, st = render_gpu(cache, p, src)
    assert st.ok, st
    ref = O.render(src, p, O.build_psf_bank(p), nat, sty)
    assert rel_err(out, ref, ref[..., :3].max()) < OUT_TOL


def test_cache_hit_and_determinism(cache):
    p = with_matrices(small_lens(spectralMode=LensDiffSpectralMode.Spectral5))
    src = S.make_frame(256, 144, 24, 1.0, 100.0, seed=8)
    a, st1 = render_gpu(cache, p, src)
    b, st2 = render_gpu(cache, p, src)
    assert st1.ok and st2.ok
    assert not st2.bank_rebuilt and not st2.spectra_rebuilt
    assert np.array_equal(a, b)
    q = p.copy(phaseDefocus=p.phaseDefocus + 1e-6)
    c, st3 = render_gpu(cache, q, src)
    assert st3.bank_rebuilt
    assert rel_err(c, a, a[..., :3].max()) < OUT_TOL


# ------------------------------------------------------------- errors ------
def test_error_behaviour_mirrors_reference(cache):
    p = with_matrices(small_lens())
    src = torch.zeros(32, 32, 4, device="cuda")
    dst = torch.zeros(32, 32, 4, device="cuda")
    stream = side_stream()
    req = image_request(src, dst, stream, frame_short_side=144)
    req.hostEnabledCudaRender = False
    err = []
    assert not run_lensdiff_cuda(req, p, cache, err)
    assert err == ["cuda-render-not-enabled-by-host"]
    req = image_request(src, dst, 0, frame_short_side=144)
    err = []
    assert not run_lensdiff_cuda(req, p, cache, err)
    assert err == ["cuda-render-not-enabled-by-host"]
    req = image_request(src, dst, stream, frame_short_side=144)
    req.dst.data = 0
    err = []
    assert not run_lensdiff_cuda(req, p, cache, err)
    assert err == ["missing-source-or-destination-cuda-buffer"]
    req = image_request(src, dst, stream, frame_short_side=144)
    st = cache.render(req, p.copy(debugView=99))
    assert not st.ok and st.stage == "invalid-debug-view"
    st = cache.render(req, p.copy(apertureMode=4))  # Custom without a decoded image: refused, never silently wrong
    assert st.code == 1 and st.stage == "custom-aperture-image-not-set"
    st = cache.render(req, p)
    assert st.ok


def test_pupil_and_basis_caches_follow_the_lens(cache):
    """The context keeps the pupil pre-pass and the DFT bases of the last
    single-lens bank while only the defocus changes.  Alternating lenses of
    different apertures and PSF windows must give each lens's own result:
    the same as a fresh context's, and the same on its second turn (to a
    float step of the frame maximum: each bank rebuild sums its statistics
    with atomics)."""
    src = S.make_frame(200, 120, 16, 1.0, 80.0, seed=21)
    pa = with_matrices(small_lens(fftForm=LensDiffFftForm.OwnChosen))
    pb = with_matrices(small_lens(fftForm=LensDiffFftForm.OwnChosen, bladeCount=9, roundness=0.6,
                                  diffractionScalePx=4.5))
    a1, st = render_gpu(cache, pa, src)
    assert st.ok, st
    b1, st = render_gpu(cache, pb, src)
    assert st.ok and st.bank_rebuilt, st
    a2, st = render_gpu(cache, pa.copy(phaseDefocus=pa.phaseDefocus + 1e-6), src)
    assert st.ok and st.bank_rebuilt, st
    a3, st = render_gpu(cache, pa, src)
    assert st.ok, st
    fresh = LensDiffPsfBankCache(0)
    try:
        b0, st = render_gpu(fresh, pb, src)
        assert st.ok, st
    finally:
        fresh.close()
    for x, y in ((a1, a3), (b1, b0)):
        assert np.abs(x - y).max() <= 1e-6 * np.abs(y[..., :3]).max()
    assert rel_err(a2, a1, a1[..., :3].max()) < OUT_TOL
    assert not np.allclose(a1, b1)
