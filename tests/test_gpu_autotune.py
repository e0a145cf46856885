"""The transforms' compiled radix orders and their autotuner.

A frame grid whose row length M and column length Py have compiled radix
orders (1920x1080 and 3840x2160 with their benchmark kernel radii: grids of
2500 x 1600 and 5000 x 3200) renders in three modes: the runtime-planned
transforms alone (-1), the first compiled order of each length (0), and the
order the autotuner times fastest on the first frame (1).  All three run the
same arithmetic up to FP32 rounding order, so they agree far inside the
output bar, and each is within that bar of the FP64 oracle.
"""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from lensdiff_b200 import synthetic as S  # noqa: E402
from lensdiff_b200.backend import LensDiffPsfBankCache, image_request  # noqa: E402
from lensdiff_b200.types import LensDiffFftForm  # noqa: E402
from oracle import check as C  # noqa: E402
from tests.helpers import OUT_TOL  # noqa: E402

pytestmark = pytest.mark.gpu


def _hd_lens():
    """The HD workload's lens on a frame with fewer highlights (same grid)."""
    p, _ = S.workload_hd()
    frame = S.make_frame(1920, 1080, 96, 1.0, 200.0, seed=77, segments=4)
    return p, frame


def _render(mode, p, frame, frames=2):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    cache = LensDiffPsfBankCache(0)
    cache.set_autotune(mode)
    stream = torch.cuda.Stream()
    src = torch.from_numpy(frame).cuda()
    dst = torch.full_like(src, -7.0)
    req = image_request(src, dst, stream, frame_short_side=p.frameShortSidePx)
    for _ in range(frames):  # the second frame runs on the tuned orders
        st = cache.render(req, p)
        assert st.ok, st
    stream.synchronize()
    assert cache.check_device_errors() == 0
    grid = st.grid_used
    choice = {n: cache.autotune_choice(n) for n in (grid[0] // 2, grid[1])}
    out = dst.cpu().numpy()
    cache.close()
    return out, grid, choice


@pytest.mark.parametrize("form", [LensDiffFftForm.OwnChosen, LensDiffFftForm.OwnFp32])
def test_radix_orders_agree_and_match_oracle(form):
    p, frame = _hd_lens()
    p = p.copy(fftForm=form)
    generic, grid, _ = _render(-1, p, frame)
    first, _, _ = _render(0, p, frame)
    tuned, _, choice = _render(1, p, frame)
    assert tuple(grid) == (2500, 1600)
    for n, c in choice.items():
        assert c is not None, f"length {n} was not tuned"
        assert math.prod(c[0]) == n and 0 <= c[1] < 8 and c[2] > 0.0
    scale = float(generic[..., :3].max())
    for other in (first, tuned):
        assert np.abs(other - generic).max() / scale < 1e-5
    ref = C.OracleResult(p, frame)
    for out in (generic, first, tuned):
        assert C.output_error(out, ref) < OUT_TOL


def test_uhd_grid_tunes_both_lengths():
    p, frame = S.workload_uhd31()
    out, grid, choice = _render(1, p, frame)
    assert tuple(grid) == (5000, 3200)
    assert choice[2500] is not None and choice[3200] is not None
    generic, _, _ = _render(-1, p, frame, frames=1)
    assert np.abs(out - generic).max() / float(generic[..., :3].max()) < 1e-5


@pytest.mark.parametrize("k", [0, 1, 2])
def test_every_compiled_order_agrees_and_matches_oracle(k):
    """Mode 2 + k pins the k-th compiled order of each length (the 1600-point
    columns have three: 25·16·4, 25·4·16 and the 16-element family's
    5·5·16·4; the 1250-point rows two, the second standing in for k = 2)."""
    p, frame = _hd_lens()
    p = p.copy(fftForm=LensDiffFftForm.OwnChosen)
    generic, grid, _ = _render(-1, p, frame)
    pinned, _, _ = _render(2 + k, p, frame)
    assert tuple(grid) == (2500, 1600)
    assert np.abs(pinned - generic).max() / float(generic[..., :3].max()) < 1e-5
    assert C.output_error(pinned, C.OracleResult(p, frame)) < OUT_TOL


def test_uhd_sixteen_element_column_order_agrees():
    """The UHD grid's 3200-point columns on the 16-element family's 5·5·16·8
    (608 threads, two CTAs per SM) against the runtime-planned transforms."""
    p, frame = S.workload_uhd31()
    pinned, grid, _ = _render(4, p, frame, frames=1)
    assert tuple(grid) == (5000, 3200)
    generic, _, _ = _render(-1, p, frame, frames=1)
    assert np.abs(pinned - generic).max() / float(generic[..., :3].max()) < 1e-5
