"""Failure detection, exercised without faulting, trapping or hanging the GPU.

Device side: every bulk-copy wait of the library is bounded, and a bulk copy
with bad arguments is refused before it is issued; ld_selftest_wait drives
both paths on purpose (a barrier nothing completes, with a short budget; a
copy of 20 bytes) and returns what the context's device error word recorded.
The context must stay usable afterwards.

Host side: an injected allocation failure (ld_inject_alloc_failure) and an
HBM budget too small for the frame come back as status codes with stage
strings, and a later call on the same context succeeds with the result of a
clean context (to the last float step of the frame maximum).
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from lensdiff_b200 import abi  # noqa: E402
from lensdiff_b200 import synthetic as S  # noqa: E402
from lensdiff_b200.backend import LensDiffPsfBankCache, image_request  # noqa: E402
from lensdiff_b200.types import LensDiffApertureMode, LensDiffFftForm, LensDiffSpectralMode  # noqa: E402
from tests.helpers import with_matrices  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cache():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    c = LensDiffPsfBankCache(0)
    yield c
    c.close()


def _lens():
    p = S.base_params(96)
    p.apertureMode = LensDiffApertureMode.Polygon
    p.bladeCount = 6
    p.pupilResolution = 128
    p.phaseDefocus = 0.2
    p.maxKernelRadiusPx = S.radius_percent(14, 96)
    p.diffractionScalePx = 3.0
    p.spectralMode = LensDiffSpectralMode.Tristimulus
    return with_matrices(p)


def _render(c, p, frame):
    stream = torch.cuda.Stream()
    src = torch.from_numpy(frame).cuda()
    dst = torch.full_like(src, -7.0)
    st = c.render(image_request(src, dst, stream, frame_short_side=p.frameShortSidePx), p)
    stream.synchronize()
    return st, dst.cpu().numpy()


def _selftest(c, mode, budget):
    word = abi.c_i32(-1)
    rc = c._lib.ld_selftest_wait(c.handle, mode, int(budget), torch.cuda.Stream().cuda_stream, ctypes.byref(word))
    return rc, int(word.value)


def test_bounded_wait_gives_up_and_context_stays_usable(cache):
    frame = S.make_frame(160, 96, 8, 1.0, 50.0, seed=3)
    st0, before = _render(cache, _lens(), frame)
    assert st0.ok, st0
    # a wait nothing completes, 2e5 SM cycles (~0.1 ms): recorded as a timeout
    rc, word = _selftest(cache, 0, 200_000)
    assert rc == abi.LD_ERR_TIMEOUT and word == 1
    assert cache.check_device_errors() == 0  # the self-test cleared the word
    st1, after = _render(cache, _lens(), frame)
    assert st1.ok, st1
    assert np.array_equal(before, after)


def test_bulk_copy_with_bad_arguments_is_refused_not_issued(cache):
    rc, word = _selftest(cache, 1, 200_000)
    assert rc == abi.LD_ERR_TIMEOUT and word == 2
    rc, word = _selftest(cache, 2, 200_000)  # a valid copy records nothing
    assert rc == abi.LD_OK and word == 0


def test_selftest_rejects_bad_modes_and_budgets(cache):
    assert _selftest(cache, 7, 200_000)[0] == abi.LD_ERR_ARG
    assert _selftest(cache, 0, 10)[0] == abi.LD_ERR_ARG
    assert _selftest(cache, 0, 10 ** 12)[0] == abi.LD_ERR_ARG


@pytest.mark.parametrize("form,afters", [(LensDiffFftForm.OwnFp32, (0, 3)),
                                         (LensDiffFftForm.OwnChosen, (0, 3, 6, 9, 12, 15))])
def test_injected_allocation_failure_is_reported_and_recoverable(form, afters):
    """Every allocation of a first render may fail; the context must then
    render the lens as a clean one does.  In the chosen form the failures
    land between the cached pre-pass, DFT basis and operand allocations, so a
    cache key recorded before its contents were written would show here."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    frame = S.make_frame(160, 96, 8, 1.0, 50.0, seed=4)
    lens = _lens().copy(fftForm=form)
    clean = LensDiffPsfBankCache(0)
    st, ref = _render(clean, lens, frame)
    clean.close()
    assert st.ok, st
    for after in afters:
        c = LensDiffPsfBankCache(0)
        assert c._lib.ld_inject_alloc_failure(c.handle, after) == abi.LD_OK
        st, _ = _render(c, lens, frame)
        if st.ok:  # fewer allocations than `after`: nothing failed
            c.close()
            continue
        assert st.code == abi.LD_ERR_OOM, st
        assert "device-allocation-failed (injected)" in st.stage
        assert c._lib.ld_inject_alloc_failure(c.handle, -1) == abi.LD_OK
        st, out = _render(c, lens, frame)
        assert st.ok, st
        # each context builds its own bank, whose ring and energy sums are
        # double-precision atomic adds in no fixed order: a sum that rounds
        # to float on the other side of a tie moves the output by one float
        # step of the frame maximum, so the bound is a few such steps
        assert np.abs(out - ref).max() <= 1e-6 * np.abs(ref[..., :3]).max()
        assert c.check_device_errors() == 0
        c.close()


def test_hbm_budget_refusal_then_a_fitting_frame():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    c = LensDiffPsfBankCache(0, hbm_budget_bytes=64 << 10)  # 64 KiB: below one 128-pixel pupil's buffers
    st, _ = _render(c, _lens(), S.make_frame(160, 96, 8, 1.0, 50.0, seed=5))
    assert st.code == abi.LD_ERR_BUDGET and "hbm-budget-exceeded" in st.stage
    c.close()
