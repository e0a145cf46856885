"""Render modes beyond the Augment composite, through the C ABI on the GPU,
against the reference's own CPU renderer (RunLensDiffCpuReference compiled
from the reference sources into oracle/_ref) and the FP64 oracle.

Preserve energy (LensDiffCpuReference.cpp:2104-2109, :2172-2178): the effect
is scaled so that its luma sum over the whole source frame equals the luma sum
of the redistributed highlights, whatever the render window; effect gain is
clamped to [0, 1] and the core compensation equals it.

The reference accumulates the two luma sums in sequential float; the GPU path
sums in FP64.  At the frame sizes here the float sums are exact to ~1e-6
relative, far below the output tolerance (2e-4 of the frame maximum).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from lensdiff_b200 import synthetic as S  # noqa: E402
from lensdiff_b200.backend import LensDiffPsfBankCache, image_request  # noqa: E402
from lensdiff_b200.types import LensDiffApertureMode, LensDiffEnergyMode, LensDiffSpectralMode  # noqa: E402
from oracle import ld_oracle as O  # noqa: E402
from oracle import ref_lib as R  # noqa: E402
from tests.helpers import OUT_TOL, golden_cases, rel_err, spectrum_matrices, with_matrices  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cache():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    c = LensDiffPsfBankCache(0)
    yield c
    c.close()


def _lens(**kw):
    p = S.base_params(144)
    p.apertureMode = LensDiffApertureMode.Polygon
    p.bladeCount = 7
    p.roundness = 0.3
    p.pupilResolution = 128
    p.phaseDefocus = 0.2
    p.phaseComaX = 0.1
    p.maxKernelRadiusPx = S.radius_percent(27, 144)
    p.diffractionScalePx = 3.0
    p.spectralMode = LensDiffSpectralMode.Tristimulus
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _render(cache, p, src, src_origin=(0, 0), dst_shape=None, dst_origin=None, render_window=None):
    stream = torch.cuda.Stream()
    s = torch.from_numpy(np.ascontiguousarray(src, np.float32)).cuda()
    d = torch.full(dst_shape or src.shape, -7.0, device="cuda", dtype=torch.float32)
    req = image_request(s, d, stream, src_origin=src_origin, dst_origin=dst_origin, render_window=render_window,
                        frame_short_side=p.frameShortSidePx)
    st = cache.render(req, p)
    torch.cuda.synchronize()
    assert st.ok, st
    assert cache.check_device_errors() == 0
    return d.cpu().numpy()


def _oracle(p, src, **kw):
    mats = () if p.spectralMode == LensDiffSpectralMode.Mono else spectrum_matrices(p)
    return O.render(src, p, O.build_psf_bank(p), *mats, **kw)


def _reference_available():
    if not R.available():
        pytest.skip("the compiled reference (oracle/_ref) is not present")


@pytest.mark.parametrize("mode,gain", [(LensDiffSpectralMode.Tristimulus, 0.8),
                                       (LensDiffSpectralMode.Mono, 1.0),
                                       (LensDiffSpectralMode.Spectral5, 0.5)])
def test_preserve_energy_matches_reference(cache, mode, gain):
    _reference_available()
    p = _lens(spectralMode=mode, energyMode=LensDiffEnergyMode.Preserve, effectGain=gain, corePreserve=0.1)
    src = S.make_frame(224, 144, 20, 1.0, 80.0, seed=11)
    out = _render(cache, with_matrices(p), src)
    ref = R.render(p, src)
    assert rel_err(out, ref, ref[..., :3].max()) < OUT_TOL
    orc = _oracle(p, src)
    assert rel_err(out, orc, orc[..., :3].max()) < OUT_TOL


def test_preserve_energy_sums_over_whole_frame_not_window(cache):
    _reference_available()
    p = _lens(energyMode=LensDiffEnergyMode.Preserve, effectGain=1.0)
    src = S.make_frame(200, 120, 16, 1.0, 60.0, seed=12)
    window = (30, 10, 150, 90)
    out = _render(cache, with_matrices(p), src, render_window=window)
    ref = R.render(p, src, render_window=window)
    x1, y1, x2, y2 = window
    assert np.all(out[:y1] == -7.0) and np.all(out[:, :x1] == -7.0)
    inside = out[y1:y2, x1:x2]
    refin = ref[y1:y2, x1:x2]
    assert rel_err(inside, refin, refin[..., :3].max()) < OUT_TOL


# ------------------------------------------------------------ field zones ----
# Field-varying aberrations (ResolveLensDiffFieldZoneParams, LensDiffPhase.cpp:
# 112-168): every zone of a 3 x 3 grid gets its own Zernike coefficients, its
# own PSF bank and its own convolution; the zone effects are blended with tent
# weights (accumulateWeightedImage, LensDiffCpuReference.cpp:1452-1475).
def _field_lens(**kw):
    from lensdiff_b200.types import LensDiffPhaseMode
    return _lens(phaseMode=LensDiffPhaseMode.Enabled, phaseFieldStrength=1.0, phaseFieldEdgeBias=0.5,
                 phaseFieldComaRadial=0.3, phaseFieldAstigTangential=0.2, phaseFieldDefocus=0.1, **kw)


@pytest.mark.parametrize("energy", [LensDiffEnergyMode.Augment, LensDiffEnergyMode.Preserve])
def test_field_zones_match_reference(cache, energy):
    _reference_available()
    p = _field_lens(energyMode=energy)
    src = S.make_frame(200, 120, 16, 1.0, 60.0, seed=13)
    out = _render(cache, with_matrices(p), src)
    ref = R.render(p, src)
    assert rel_err(out, ref, ref[..., :3].max()) < OUT_TOL
    # the zones matter: without them the result is measurably different
    flat = R.render(p.copy(phaseFieldStrength=0.0), src)
    assert rel_err(flat, ref, ref[..., :3].max()) > 20 * OUT_TOL


def test_field_zones_cached_and_window(cache):
    _reference_available()
    p = _field_lens(spectralMode=LensDiffSpectralMode.Mono)
    src = S.make_frame(180, 110, 12, 1.0, 50.0, seed=14)
    window = (20, 15, 160, 100)
    first = _render(cache, with_matrices(p), src, render_window=window)
    again = _render(cache, with_matrices(p), src, render_window=window)  # all nine zones cached
    assert np.array_equal(first, again)
    ref = R.render(p, src, render_window=window)
    x1, y1, x2, y2 = window
    assert rel_err(first[y1:y2, x1:x2], ref[y1:y2, x1:x2], ref[y1:y2, x1:x2, :3].max()) < OUT_TOL


def test_field_grid_8x8_matches_oracle(cache):
    """The 8 x 8 zone grid of the batching workload (an extension: the
    reference's grid is 3 x 3), against the FP64 oracle restated from the
    same zone rules."""
    p = _field_lens(fieldGrid=8, pupilResolution=64, maxKernelRadiusPx=S.radius_percent(12, 144))
    src = S.make_frame(160, 96, 10, 1.0, 40.0, seed=15)
    out = _render(cache, with_matrices(p), src)
    orc = _oracle(p, src, field_grid=8)
    assert rel_err(out, orc, orc[..., :3].max()) < OUT_TOL


def test_field_grid_8x8_chosen_form_batched_windows(cache):
    """With the chosen form, the 64 zones' PSF windows come from one batched
    launch per pass of the persistent tensor-core GEMM; the frame still meets
    the oracle, and a second frame that changes one zone coefficient rebuilds
    every zone through the batch again."""
    from lensdiff_b200.types import LensDiffFftForm
    p = _field_lens(fieldGrid=8, pupilResolution=64, maxKernelRadiusPx=S.radius_percent(12, 144),
                    fftForm=LensDiffFftForm.OwnChosen)
    src = S.make_frame(160, 96, 10, 1.0, 40.0, seed=16)
    for q in (p, p.copy(phaseFieldComaRadial=0.35)):
        out = _render(cache, with_matrices(q), src)
        orc = _oracle(q.copy(fftForm=LensDiffFftForm.OwnFp32), src, field_grid=8)
        assert rel_err(out, orc, orc[..., :3].max()) < OUT_TOL


# ------------------------------------------------------- cuFFT comparator ----
# fft_form LD_FFT_CUFFT runs the same bank and frame chain with cuFFT doing the
# transforms (the library the reference CUDA backend uses); it is the timing
# comparator and must meet the same parity bar.
@pytest.mark.parametrize("mode,energy", [(LensDiffSpectralMode.Tristimulus, LensDiffEnergyMode.Augment),
                                         (LensDiffSpectralMode.Mono, LensDiffEnergyMode.Augment),
                                         (LensDiffSpectralMode.Spectral5, LensDiffEnergyMode.Preserve)])
def test_cufft_form_matches_reference(cache, mode, energy):
    from lensdiff_b200.types import LensDiffFftForm
    _reference_available()
    p = _lens(spectralMode=mode, energyMode=energy, chromaticFocus=0.3)
    src = S.make_frame(224, 144, 20, 1.0, 80.0, seed=16)
    own = _render(cache, with_matrices(p), src)
    cuf = _render(cache, with_matrices(p.copy(fftForm=LensDiffFftForm.Cufft)), src)
    ref = R.render(p, src)
    scale = ref[..., :3].max()
    assert rel_err(cuf, ref, scale) < OUT_TOL
    assert rel_err(own, ref, scale) < OUT_TOL


def test_cufft_form_rejects_field_zones(cache):
    from lensdiff_b200.types import LensDiffFftForm
    p = _field_lens(fftForm=LensDiffFftForm.Cufft)
    src = S.make_frame(64, 48, 4, 1.0, 10.0, seed=17)
    stream = torch.cuda.Stream()
    s = torch.from_numpy(src).cuda()
    d = torch.zeros_like(s)
    st = cache.render(image_request(s, d, stream, frame_short_side=p.frameShortSidePx), with_matrices(p))
    assert not st.ok and "field-zones" in st.stage


# ------------------------------------------------------------ CUDA graphs ----
def test_graph_replay_matches_direct_launches(cache):
    """Per-frame chains are captured into CUDA graphs and replayed for frames
    with identical launches (same buffers); replayed frames read their new
    contents and equal directly launched ones bit for bit."""
    p = with_matrices(_lens())
    frames = [S.make_frame(240, 136, 16, 1.0, 60.0, seed=s) for s in (31, 32, 33)]
    stream = torch.cuda.Stream()
    s = torch.empty(frames[0].shape, device="cuda", dtype=torch.float32)
    d = torch.empty_like(s)
    req = image_request(s, d, stream, frame_short_side=p.frameShortSidePx)

    def run(frame):
        s.copy_(torch.from_numpy(frame))
        torch.cuda.synchronize()
        st = cache.render(req, p)
        torch.cuda.synchronize()
        assert st.ok, st
        return d.cpu().numpy()

    cache.set_graphs(False)
    direct = [run(f) for f in frames]
    cache.set_graphs(True)
    try:
        replayed = [run(f) for f in frames + frames]  # capture once, then replay
    finally:
        cache.set_graphs(True)
    for i, out in enumerate(replayed):
        assert np.array_equal(out, direct[i % 3]), i
    assert cache.check_device_errors() == 0


# ------------------------------------------------------------ chosen form ----
# fft_form LD_FFT_OWN_CHOSEN stores the kernel spectra and the column-pass
# outputs in FP16 with one float scale per spectrum column (half the bytes of
# the largest frame arrays), and builds the PSF windows by DFT-as-GEMM on the
# tensor cores (BF16 3-way split, FP32 accumulation); it must meet the same
# bars: the bank kernels against the reference's golden fixtures within 1e-4
# of their peak, the output within 2e-4 of the frame maximum.
@pytest.mark.parametrize("name", sorted(golden_cases().keys()))
def test_chosen_form_bank_matches_reference_fixture(cache, name):
    from lensdiff_b200.types import LensDiffFftForm, LensDiffLookMode
    from tests.helpers import PSF_TOL, golden_case
    p, _, _, bank, wl, meta = golden_case(name)
    p = p.copy(fftForm=LensDiffFftForm.OwnChosen)
    if p.lookMode != LensDiffLookMode.Physical:
        p = p.copy(lookMode=LensDiffLookMode.Physical, energyMode=1)
    wls, kernels, st = cache.export_psf_bank(p, torch.cuda.current_stream())
    assert st.ok, st
    assert cache.check_device_errors() == 0
    assert st.support_radius == meta["support_radius"]
    for k, ref in zip(kernels, bank):
        assert k.shape == ref.shape
        assert rel_err(k, ref, ref.max()) < PSF_TOL


def test_chosen_form_bank_large_pupil_matches_fp32_form(cache):
    """Pupil 512 -> PSF 2048 with 31 wavelengths (the UHD bank's sizes, several
    128-column tiles per window): the tensor-core bank against the FP32 FFT bank."""
    from lensdiff_b200.types import LensDiffFftForm
    from tests.helpers import PSF_TOL
    p, _ = S.workload_uhd31()
    _, k32, st = cache.export_psf_bank(p, torch.cuda.current_stream())
    assert st.ok, st
    _, kch, st = cache.export_psf_bank(p.copy(fftForm=LensDiffFftForm.OwnChosen), torch.cuda.current_stream())
    assert st.ok, st
    assert cache.check_device_errors() == 0
    assert len(kch) == 31
    for a, b in zip(kch, k32):
        assert a.shape == b.shape
        assert rel_err(a, b, b.max()) < PSF_TOL
@pytest.mark.parametrize("kw", [{}, {"spectralMode": LensDiffSpectralMode.Spectral9, "chromaticFocus": 0.3},
                                {"energyMode": LensDiffEnergyMode.Preserve},
                                {"spectralMode": LensDiffSpectralMode.Mono}])
def test_chosen_form_matches_reference(cache, kw):
    from lensdiff_b200.types import LensDiffFftForm
    _reference_available()
    p = _lens(**kw)
    src = S.make_frame(256, 144, 24, 1.0, 1000.0, seed=18)
    out = _render(cache, with_matrices(p.copy(fftForm=LensDiffFftForm.OwnChosen)), src)
    ref = R.render(p, src)
    assert rel_err(out, ref, ref[..., :3].max()) < OUT_TOL


def test_chosen_form_field_zones(cache):
    from lensdiff_b200.types import LensDiffFftForm
    _reference_available()
    p = _field_lens()
    src = S.make_frame(200, 120, 16, 1.0, 300.0, seed=19)
    out = _render(cache, with_matrices(p.copy(fftForm=LensDiffFftForm.OwnChosen)), src)
    ref = R.render(p, src)
    assert rel_err(out, ref, ref[..., :3].max()) < OUT_TOL


# ------------------------------------------------------------- Split look ----
# Core (azimuthal mean) and structure (positive residual) kernels convolved
# separately, each spectrally mapped, soft-shouldered and weighted
# (LensDiffCpuReference.cpp:2123-2146, :1631-1645, :84-90, :1340-1368).
@pytest.mark.parametrize("kw", [
    {"spectralMode": LensDiffSpectralMode.Tristimulus},
    {"spectralMode": LensDiffSpectralMode.Mono, "coreShoulder": 0.0},
    {"spectralMode": LensDiffSpectralMode.Spectral9, "energyMode": LensDiffEnergyMode.Preserve,
     "anisotropyEmphasis": 0.3},
])
def test_split_look_matches_reference(cache, kw):
    from lensdiff_b200.types import LensDiffLookMode
    _reference_available()
    p = _lens(lookMode=LensDiffLookMode.Split, coreGain=0.8, structureGain=1.4, coreShoulder=2.0,
              structureShoulder=0.5, **{k: v for k, v in kw.items() if k != "coreShoulder"})
    if "coreShoulder" in kw:
        p = p.copy(coreShoulder=kw["coreShoulder"])
    src = S.make_frame(224, 144, 20, 1.0, 80.0, seed=51)
    out = _render(cache, with_matrices(p), src)
    ref = R.render(p, src)
    assert rel_err(out, ref, ref[..., :3].max()) < OUT_TOL
    phys = R.render(p.copy(lookMode=LensDiffLookMode.Physical), src)
    assert rel_err(phys, ref, ref[..., :3].max()) > 20 * OUT_TOL  # the look matters here


def test_split_render_after_physical_render_of_the_same_lens(cache):
    """A Physical render builds the bank with the shaping statistics taken in
    the lambda-rescale (anisotropy gain 1), without the ring means; a Split
    render of the same lens then reuses that bank and computes its ring means
    from the canvas."""
    from lensdiff_b200.types import LensDiffFftForm, LensDiffLookMode
    _reference_available()
    src = S.make_frame(224, 144, 20, 1.0, 80.0, seed=53)
    for form in (LensDiffFftForm.OwnFp32, LensDiffFftForm.OwnChosen):
        p = _lens(phaseDefocus=0.23, coreGain=0.8, structureGain=1.4, coreShoulder=2.0, structureShoulder=0.5,
                  fftForm=form)
        phys = _render(cache, with_matrices(p), src)
        ref_phys = R.render(p, src)
        assert rel_err(phys, ref_phys, ref_phys[..., :3].max()) < OUT_TOL, form
        q = p.copy(lookMode=LensDiffLookMode.Split)
        out = _render(cache, with_matrices(q), src)
        ref = R.render(q, src)
        assert rel_err(out, ref, ref[..., :3].max()) < OUT_TOL, form


@pytest.mark.parametrize("emphasis", [0.0, 0.3, 1.0])
def test_bank_with_anisotropy_emphasis_matches_reference(cache, emphasis):
    """Gain 1 (emphasis 0) takes the fused path; gains 2.2 and 5 the separate
    shaping pass (reshapeAnisotropy, LensDiffCpuReference.cpp:1122-1134)."""
    from lensdiff_b200.types import LensDiffFftForm
    from tests.helpers import PSF_TOL
    _reference_available()
    p = _lens(anisotropyEmphasis=emphasis, spectralMode=LensDiffSpectralMode.Spectral5)
    _, ref, _, _, _ = R.bank(p)
    for form in (LensDiffFftForm.OwnFp32, LensDiffFftForm.OwnChosen):
        wls, kernels, st = cache.export_psf_bank(p.copy(fftForm=form), torch.cuda.current_stream())
        assert st.ok, st
        assert len(kernels) == len(ref)
        for k, r in zip(kernels, ref):
            assert k.shape == r.shape, (form, k.shape, r.shape)
            assert rel_err(k, r, r.max()) < PSF_TOL, form


def test_split_look_with_field_zones_and_chosen_form(cache):
    from lensdiff_b200.types import LensDiffFftForm, LensDiffLookMode
    _reference_available()
    p = _field_lens(lookMode=LensDiffLookMode.Split, coreGain=1.0, structureGain=1.2, structureShoulder=1.0)
    src = S.make_frame(200, 120, 16, 1.0, 60.0, seed=52)
    ref = R.render(p, src)
    for form in (LensDiffFftForm.OwnFp32, LensDiffFftForm.OwnChosen):
        out = _render(cache, with_matrices(p.copy(fftForm=form)), src)
        assert rel_err(out, ref, ref[..., :3].max()) < OUT_TOL, form


# ---------------------------------------------------------- aperture modes ---
# Star, spiral, square-grid and snowflake apertures (LensDiffCpuReference.cpp:
# 509-668, :758-822) against the compiled reference: the raw PSF (after an
# exact renormalisation: the reference normalises with a sequential float
# sum) and the rendered frame.
@pytest.mark.parametrize("mode,blades,rnd", [(2, 5, 0.3), (3, 4, 0.6), (6, 5, 0.2), (7, 8, 0.5)])
def test_aperture_modes_match_reference(cache, mode, blades, rnd):
    from tests.helpers import PSF_TOL
    _reference_available()
    p = _lens(apertureMode=LensDiffApertureMode(mode), bladeCount=blades, roundness=rnd, rotationDeg=12.0,
              centralObstruction=0.1, pupilResolution=256)
    from lensdiff_b200.backend import resolve_sizes
    np_, S_, _, _ = resolve_sizes(p)
    out = torch.zeros(S_, S_, device="cuda")
    st = cache.raw_psf(p, 1, out, torch.cuda.Stream())
    assert st.ok, st
    torch.cuda.synchronize()
    got = out.cpu().numpy().astype(np.float64)
    ref = R.raw_psf(p, 550.0).astype(np.float64)
    got /= got.sum()
    ref /= ref.sum()
    assert rel_err(got, ref, ref.max()) < PSF_TOL
    src = S.make_frame(200, 120, 14, 1.0, 60.0, seed=60 + mode)
    img = _render(cache, with_matrices(p), src)
    refimg = R.render(p, src)
    assert rel_err(img, refimg, refimg[..., :3].max()) < OUT_TOL


# ------------------------------------- scatter, creative fringe, working frame ---
# After the effect (LensDiffCpuReference.cpp:2180-2198): scatter adds
# amount * (effect convolved with a normalised Gaussian, :1680-1700); the
# creative fringe samples red and blue bilinearly at +/- a radial shift
# (:1499-1534); resolution-aware rendering computes the effect on the source
# resampled to a 2160-pixel short side and resamples the redistributed source
# and the effect back (:2089-2094, :2192-2196, :414-434).
@pytest.mark.parametrize("kw", [
    {"scatterAmount": 0.5, "scatterRadius": 10.0},
    {"scatterAmount": 0.8, "scatterRadius": 4.0, "spectralMode": LensDiffSpectralMode.Mono},
    {"scatterAmount": 0.3, "scatterRadius": 25.0, "energyMode": LensDiffEnergyMode.Preserve,
     "spectralMode": LensDiffSpectralMode.Spectral5},
    {"creativeFringe": 2.0},
    {"creativeFringe": 1.0, "scatterAmount": 0.4, "scatterRadius": 6.0, "spectralMode": LensDiffSpectralMode.Mono},
])
def test_scatter_and_fringe_match_reference(cache, kw):
    _reference_available()
    p = _lens(**kw)
    src = S.make_frame(224, 144, 20, 1.0, 80.0, seed=71)
    out = _render(cache, with_matrices(p), src)
    ref = R.render(p, src)
    assert rel_err(out, ref, ref[..., :3].max()) < OUT_TOL
    plain = R.render(p.copy(scatterAmount=0.0, creativeFringe=0.0), src)
    assert rel_err(plain, ref, ref[..., :3].max()) > 5 * OUT_TOL  # the step matters here


def _aware_lens(short_side, **kw):
    # percentages of the 2160-pixel optics short side
    return _lens(resolutionAware=True, frameShortSidePx=short_side, maxKernelRadiusPx=S.radius_percent(30, 2160),
                 diffractionScalePx=3.0 * 144 / 2160, **kw)


@pytest.mark.parametrize("short_side,kw", [
    (1080, {}),
    (4320, {"spectralMode": LensDiffSpectralMode.Mono}),
    (1440, {"scatterAmount": 0.4, "scatterRadius": 0.5, "creativeFringe": 0.1}),
    (2880, {"energyMode": LensDiffEnergyMode.Preserve, "creativeFringe": 0.08,
            "spectralMode": LensDiffSpectralMode.Spectral5}),
])
def test_resolution_aware_matches_reference(cache, short_side, kw):
    _reference_available()
    p = _aware_lens(short_side, **kw)
    src = S.make_frame(224, 144, 20, 1.0, 80.0, seed=72)
    out = _render(cache, with_matrices(p), src)
    ref = R.render(p, src)
    assert rel_err(out, ref, ref[..., :3].max()) < OUT_TOL
    orc = _oracle(p, src)
    assert rel_err(out, orc, orc[..., :3].max()) < OUT_TOL


def test_resolution_aware_window_and_origins(cache):
    _reference_available()
    p = _aware_lens(1080, scatterAmount=0.3, scatterRadius=0.6)
    src = S.make_frame(200, 120, 16, 1.0, 60.0, seed=73)
    window = (30, 10, 150, 90)
    out = _render(cache, with_matrices(p), src, render_window=window)
    ref = R.render(p, src, render_window=window)
    x1, y1, x2, y2 = window
    assert np.all(out[:y1] == -7.0) and np.all(out[:, :x1] == -7.0)
    assert rel_err(out[y1:y2, x1:x2], ref[y1:y2, x1:x2], ref[y1:y2, x1:x2, :3].max()) < OUT_TOL


def test_post_effects_with_field_zones_split_and_chosen_form(cache):
    from lensdiff_b200.types import LensDiffFftForm, LensDiffLookMode
    _reference_available()
    p = _field_lens(lookMode=LensDiffLookMode.Split, coreGain=1.0, structureGain=1.2, structureShoulder=1.0,
                    scatterAmount=0.5, scatterRadius=8.0, creativeFringe=1.5)
    src = S.make_frame(200, 120, 16, 1.0, 60.0, seed=74)
    ref = R.render(p, src)
    for form in (LensDiffFftForm.OwnFp32, LensDiffFftForm.OwnChosen):
        out = _render(cache, with_matrices(p.copy(fftForm=form)), src)
        assert rel_err(out, ref, ref[..., :3].max()) < OUT_TOL, form


def test_post_effects_graph_replay(cache):
    """A second frame with the same settings replays the captured chain
    (scatter and composite included) and still follows its own source."""
    _reference_available()
    p = _aware_lens(1440, scatterAmount=0.4, scatterRadius=0.5, creativeFringe=0.1)
    for seed in (75, 76):
        src = S.make_frame(224, 144, 20, 1.0, 80.0, seed=seed)
        out = _render(cache, with_matrices(p), src)
        ref = R.render(p, src)
        assert rel_err(out, ref, ref[..., :3].max()) < OUT_TOL


def test_post_effects_refused_with_cufft_form(cache):
    from lensdiff_b200.types import LensDiffFftForm
    p = _lens(scatterAmount=0.5, scatterRadius=10.0, fftForm=LensDiffFftForm.Cufft)
    stream = torch.cuda.Stream()
    s = torch.zeros(64, 64, 4, device="cuda")
    d = torch.zeros_like(s)
    st = cache.render(image_request(s, d, stream), with_matrices(p))
    assert not st.ok and st.stage == "unsupported-scatter-fringe-or-resolution-aware-with-cufft-form"


# ------------------------------------------- PSF sizes with a prime factor > 5 ---
# S = 4 R_max = 1204 = 4 * 7 * 43: the reference transforms it with Bluestein's
# algorithm (LensDiffCpuReference.cpp:234-275); here the raw PSF's window (and
# the whole S x S PSF for the raw-PSF export) comes from the tensor-core DFT,
# and the first-zero calibration profiles a window around the centre.
def _bluestein_lens(**kw):
    p = _lens(pupilResolution=64, maxKernelRadiusPx=S.radius_percent(301, 144), diffractionScalePx=2.0, **kw)
    from lensdiff_b200.backend import resolve_sizes
    assert resolve_sizes(p)[1] == 1204
    return p


@pytest.mark.parametrize("form", [0, 1])
def test_non_smooth_psf_size_bank_matches_reference(cache, form):
    from lensdiff_b200.types import LensDiffFftForm
    from tests.helpers import PSF_TOL
    _reference_available()
    p = _bluestein_lens(fftForm=LensDiffFftForm(form))
    wls, kernels, st = cache.export_psf_bank(p, torch.cuda.current_stream())
    assert st.ok, st
    assert cache.check_device_errors() == 0
    rwl, rfull, _, _, rsup = R.bank(p)
    assert st.support_radius == rsup
    for k, ref in zip(kernels, rfull):
        assert k.shape == ref.shape
        assert rel_err(k, ref, ref.max()) < PSF_TOL


def test_non_smooth_psf_size_raw_psf_and_render(cache):
    from tests.helpers import PSF_TOL
    _reference_available()
    p = _bluestein_lens()
    out = torch.zeros(1204, 1204, device="cuda")
    st = cache.raw_psf(p, 1, out, torch.cuda.Stream())
    assert st.ok, st
    torch.cuda.synchronize()
    got = out.cpu().numpy().astype(np.float64)
    ref = R.raw_psf(p, 550.0).astype(np.float64)
    got /= got.sum()
    ref /= ref.sum()
    assert rel_err(got, ref, ref.max()) < PSF_TOL
    src = S.make_frame(200, 120, 14, 1.0, 60.0, seed=81)
    img = _render(cache, with_matrices(p), src)
    refimg = R.render(p, src)
    assert rel_err(img, refimg, refimg[..., :3].max()) < OUT_TOL


# ------------------------------------------------ DaVinci Intermediate transfer ---
# The source is decoded to linear as it is read and the output encoded back
# (loadSourceRgba, LensDiffCpuReference.cpp:174-192; :2248-2250), in every
# transform form and with the resolution-aware working frame.
@pytest.mark.parametrize("kw", [{"fftForm": 0}, {"fftForm": 1}, {"fftForm": 2},
                                {"fftForm": 0, "energyMode": LensDiffEnergyMode.Preserve, "creativeFringe": 1.0},
                                {"fftForm": 1, "resolutionAware": True, "frameShortSidePx": 1080,
                                 "maxKernelRadiusPx": 1.25, "diffractionScalePx": 0.2}])
def test_davinci_transfer_matches_reference(cache, kw):
    from lensdiff_b200.types import LensDiffFftForm
    _reference_available()
    kw = dict(kw)
    form = LensDiffFftForm(kw.pop("fftForm"))
    p = _lens(inputTransfer=1, **kw)
    src = S.make_frame(224, 144, 20, 0.55, 0.8, seed=91)
    out = _render(cache, with_matrices(p.copy(fftForm=form)), src)
    ref = R.render(p, src)
    # the output bar is on linear RGB: compare the decoded frames (the log
    # curve's slope is 10.4 near black, so encoded differences of the FP16
    # chosen form exceed the bar there while the linear ones stay within it)
    lin, rlin = O.davinci_decode(out[..., :3]), O.davinci_decode(ref[..., :3])
    assert rel_err(lin, rlin, rlin.max()) < OUT_TOL
    if form != LensDiffFftForm.OwnChosen:
        assert rel_err(out, ref, ref[..., :3].max()) < OUT_TOL


# ------------------------------------------------------ frame debug views ---
# renderDebugView (LensDiffCpuReference.cpp:1789-1824): the selection mask over
# its maximum, the core / structure / final effects, the scatter and creative
# fringe previews, resampled to the source frame when resolution-aware;
# unencoded, alpha 1.
_DV = {"selection": 1, "core": 5, "structure": 6, "effect": 7, "fringe": 12, "scatter": 13}


@pytest.mark.parametrize("view,kw", [
    ("selection", {}),
    ("selection", {"resolutionAware": True, "frameShortSidePx": 1080, "maxKernelRadiusPx": 1.25,
                   "diffractionScalePx": 0.2}),
    ("effect", {"energyMode": LensDiffEnergyMode.Preserve, "scatterAmount": 0.5, "scatterRadius": 8.0,
                "creativeFringe": 1.5}),
    ("core", {}),
    ("structure", {}),
    ("core", {"lookMode": 1, "coreShoulder": 2.0, "coreGain": 0.7, "spectralMode": LensDiffSpectralMode.Spectral5}),
    ("structure", {"lookMode": 1, "structureShoulder": 0.5, "structureGain": 1.3,
                   "spectralMode": LensDiffSpectralMode.Mono}),
    ("scatter", {"scatterAmount": 0.5, "scatterRadius": 8.0, "energyMode": LensDiffEnergyMode.Preserve}),
    ("scatter", {}),
    ("fringe", {"creativeFringe": 2.0, "scatterAmount": 0.3, "scatterRadius": 6.0}),
    ("fringe", {}),
    ("fringe", {"creativeFringe": 0.1, "resolutionAware": True, "frameShortSidePx": 1440,
                "maxKernelRadiusPx": 1.25, "diffractionScalePx": 0.2}),
])
def test_frame_debug_views_match_reference(cache, view, kw):
    _reference_available()
    p = _lens(debugView=_DV[view], **kw)
    src = S.make_frame(224, 144, 20, 1.0, 80.0, seed=95)
    out = _render(cache, with_matrices(p), src)
    ref = R.render(p, src)
    scale = max(float(ref[..., :3].max()), 1e-30)
    assert rel_err(out, ref, scale) < OUT_TOL
    assert np.all(out[..., 3] == 1.0)


def test_frame_debug_view_with_field_zones_and_window(cache):
    _reference_available()
    p = _field_lens(debugView=_DV["core"])
    src = S.make_frame(200, 120, 16, 1.0, 60.0, seed=96)
    window = (30, 10, 150, 90)
    out = _render(cache, with_matrices(p), src, render_window=window)
    ref = R.render(p, src, render_window=window)
    x1, y1, x2, y2 = window
    assert np.all(out[:y1] == -7.0)
    assert rel_err(out[y1:y2, x1:x2], ref[y1:y2, x1:x2], ref[y1:y2, x1:x2, :3].max()) < OUT_TOL


# ----------------------------------------------------- static debug views ---
# BuildLensDiffStaticDebugRgba (LensDiffCpuReference.cpp:1909-1970): the
# pupil, PSF, OTF, phase, field-edge phase and PSF, and chromatic split drawn
# into the centred square of the frame (values in [0, 1]).
@pytest.mark.parametrize("view,kw", [
    ("pupil", {}), ("psf", {}), ("otf", {}), ("phase", {}), ("split", {}),
    ("phase_edge", {}), ("field_psf", {}),
    ("phase_edge", {"field": True}), ("field_psf", {"field": True}),
    ("psf", {"spectralMode": LensDiffSpectralMode.Mono, "apertureMode": LensDiffApertureMode(3), "bladeCount": 6}),
    ("split", {"spectralMode": LensDiffSpectralMode.Spectral9, "chromaticSpread": 0.3}),
    ("phase", {"pupilDecenterX": 0.1, "centralObstruction": 0.25, "vaneCount": 3, "vaneThickness": 0.05}),
])
def test_static_debug_views_match_reference(cache, view, kw):
    _reference_available()
    ids = {"pupil": 2, "psf": 3, "otf": 4, "phase": 8, "phase_edge": 9, "field_psf": 10, "split": 11}
    kw = dict(kw)
    field = kw.pop("field", False)
    p = (_field_lens if field else _lens)(debugView=ids[view], **kw)
    src = S.make_frame(224, 144, 20, 1.0, 80.0, seed=97)
    out = _render(cache, with_matrices(p), src)
    ref = R.render(p, src)
    assert rel_err(out, ref, 1.0) < OUT_TOL
    assert float(ref[..., :3].max()) > 0.5  # the view draws something


def test_static_debug_view_window_and_origins(cache):
    _reference_available()
    p = _lens(debugView=4)
    src = S.make_frame(200, 120, 16, 1.0, 60.0, seed=98)
    window = (30, 10, 150, 90)
    out = _render(cache, with_matrices(p), src, render_window=window)
    ref = R.render(p, src, render_window=window)
    x1, y1, x2, y2 = window
    assert np.all(out[:y1] == -7.0) and np.all(out[:, :x1] == -7.0)
    assert rel_err(out[y1:y2, x1:x2], ref[y1:y2, x1:x2], 1.0) < OUT_TOL
