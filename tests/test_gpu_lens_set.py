"""Banks of several unrelated lenses built together (ld_build_psf_banks):
pupil size, PSF size (5-smooth and not), wavelength count and phase all
differ between the lenses, and their tensor-core windows come from one
persistent GEMM launch per transform pass.

Each bank must equal the bank EnsureLensDiffPsfBank builds for that lens
alone (LensDiffCpuReference.cpp:2068-2071): against the FP64 oracle within
1e-4 of the kernel's peak, and against the same lens's single-bank build on
the GPU within 1e-6 (the two runs differ only in the order of the FP64 atomic
ring sums).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from lensdiff_b200 import synthetic as S  # noqa: E402
from lensdiff_b200.backend import LensDiffPsfBankCache, image_request  # noqa: E402
from lensdiff_b200.types import LensDiffFftForm  # noqa: E402
from oracle import ld_oracle as O  # noqa: E402
from tests.helpers import PSF_TOL, rel_err  # noqa: E402

pytestmark = pytest.mark.gpu

SAME_TOL = 1e-6


@pytest.fixture(scope="module")
def cache():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    c = LensDiffPsfBankCache(0)
    yield c
    c.close()


def _lenses():
    """Four lenses: PSF sizes 524 (4 x 131, not 5-smooth), 600, 512 and 640;
    pupils 64-128; 3, 5, 9 and 16 wavelengths."""
    ps = S.lens_instances(4, seed=77, pupil=(64, 128), pad=(2.0, 4.0), bins=(3, 9))
    radii = (131, 150, 96, 160)
    bins = (3, 5, 9, 16)
    for p, r, b in zip(ps, radii, bins):
        p.maxKernelRadiusPx = S.radius_percent(r, 2160)
        p.wavelengthsNm = [float(v) for v in np.linspace(400.0, 700.0, b)]
    return ps


def _export(c, p):
    wls, kernels, st = c.export_psf_bank(p, torch.cuda.current_stream())
    assert st.ok, st
    return kernels, st


def test_lens_set_matches_single_builds_and_oracle(cache):
    ps = _lenses()
    sizes = [O.resolve_sizes(p) for p in ps]
    assert len({s[1] for s in sizes}) == 4  # four PSF sizes
    st = cache.build_psf_banks(ps, torch.cuda.current_stream())
    assert st.ok, st
    assert st.banks_rebuilt == 4
    assert cache.check_device_errors() == 0
    from_set = []
    for p in ps:
        k, est = _export(cache, p)
        assert not est.bank_rebuilt  # found among the set's banks
        from_set.append(k)
    # each lens alone, in a second context
    single = LensDiffPsfBankCache(0)
    try:
        for p, ks in zip(ps, from_set):
            kb, _ = _export(single, p)
            assert len(kb) == len(ks)
            for a, b in zip(ks, kb):
                assert a.shape == b.shape
                assert rel_err(a, b, b.max()) < SAME_TOL
    finally:
        single.close()
    for i in (0, 2):  # the FP64 oracle for the non-smooth and the smallest PSF
        ob = O.build_psf_bank(ps[i])
        assert len(from_set[i]) == len(ob.bins)
        for k, b in zip(from_set[i], ob.bins):
            assert k.shape == b.full.shape
            assert rel_err(k, b.full, b.full.max()) < PSF_TOL


def test_lens_set_large_pupils(cache):
    """Pupils of 1000 and 1024 (28 K-chunks per GEMM tile): PSF 4000 against
    the FP32 FFT bank of the same lens, PSF 4124 (4 x 1031) against the FP64
    oracle."""
    ps = S.lens_instances(2, seed=78, pupil=(1000, 1000), bins=(8, 8))
    ps[1] = S.lens_instances(1, seed=79, pupil=(1024, 1024), bins=(4, 4))[0]
    ps[0].maxKernelRadiusPx = S.radius_percent(1000, 2160)
    ps[1].maxKernelRadiusPx = S.radius_percent(1031, 2160)
    assert [O.resolve_sizes(p)[1] for p in ps] == [4000, 4124]
    st = cache.build_psf_banks(ps, torch.cuda.current_stream())
    assert st.ok, st
    assert cache.check_device_errors() == 0
    k0, _ = _export(cache, ps[0])
    k1, _ = _export(cache, ps[1])
    single = LensDiffPsfBankCache(0)
    try:
        kf, _ = _export(single, ps[0].copy(fftForm=LensDiffFftForm.OwnFp32))
    finally:
        single.close()
    for a, b in zip(k0, kf):
        assert a.shape == b.shape
        assert rel_err(a, b, b.max()) < PSF_TOL
    ob = O.build_psf_bank(ps[1])
    for a, b in zip(k1, ob.bins):
        assert a.shape == b.full.shape
        assert rel_err(a, b.full, b.full.max()) < PSF_TOL


def test_lens_set_keeps_unchanged_banks_and_mixes_forms(cache):
    ps = _lenses()
    st = cache.build_psf_banks(ps, torch.cuda.current_stream())
    assert st.ok, st
    # lens 1 changes; lens 2 moves to the FP32 FFT form (S = 512, built on
    # its own); lenses 0 and 3 are kept
    ps[1] = ps[1].copy(phaseDefocus=0.3)
    ps[2] = ps[2].copy(fftForm=LensDiffFftForm.OwnFp32)
    st = cache.build_psf_banks(ps, torch.cuda.current_stream())
    assert st.ok, st
    assert st.banks_rebuilt == 2
    for i in (1, 2):
        k, _ = _export(cache, ps[i])
        ob = O.build_psf_bank(ps[i])
        for a, b in zip(k, ob.bins):
            assert rel_err(a, b.full, b.full.max()) < PSF_TOL
    assert cache.check_device_errors() == 0


def test_render_uses_a_set_bank(cache):
    ps = _lenses()
    st = cache.build_psf_banks(ps, torch.cuda.current_stream())
    assert st.ok, st
    p = ps[3].copy(frameShortSidePx=2160)
    h, w = 96, 128
    src = torch.from_numpy(S.make_frame(w, h, 6, 1.0, 50.0, seed=5)).cuda()
    dst = torch.zeros_like(src)
    s = torch.cuda.Stream()  # the plugin refuses the null stream (LensDiffCuda.cu:4646-4657)
    st = cache.render(image_request(src, dst, s, frame_short_side=2160), p)
    torch.cuda.synchronize()
    assert st.ok, st
    assert not st.bank_rebuilt
    single = LensDiffPsfBankCache(0)
    try:
        ref = torch.zeros_like(src)
        st2 = single.render(image_request(src, ref, s, frame_short_side=2160), p)
        torch.cuda.synchronize()
        assert st2.ok, st2
        assert st2.bank_rebuilt
        a, b = dst.cpu().numpy(), ref.cpu().numpy()
        assert rel_err(a, b, np.abs(b[..., :3]).max()) < SAME_TOL
    finally:
        single.close()


def test_lens_set_rejects_bad_arguments(cache):
    st = cache.build_psf_banks([], torch.cuda.current_stream())
    assert not st.ok and st.stage == "invalid-lens-count"
    bad = _lenses()[:2]
    bad[1] = bad[1].copy(apertureMode=4)  # Custom aperture with no decoded image handed over
    st = cache.build_psf_banks(bad, torch.cuda.current_stream())
    assert not st.ok and st.stage == "custom-aperture-image-not-set"
