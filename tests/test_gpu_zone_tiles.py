"""Overlap-add tiles for field zones, against the FP64 oracle.

A zone's tent weight (accumulateWeightedImage, LensDiffCpuReference.cpp:
1452-1475) is zero beyond its neighbours' centres, so on a fine zone grid each
zone convolves only its window plus the kernel's reach, on one tile-sized FFT
grid shared by every zone, instead of the whole frame (taken when that grid
is at most half the frame's).  The tile's grid origin lies up to a kernel
radius outside the frame at the borders; pixels there read as zero.  Every
render below takes the tiled path (the status reports the tile grid) and must
match the oracle, which convolves each zone over the whole frame.
"""
import pytest

torch = pytest.importorskip("torch")

from lensdiff_b200 import synthetic as S  # noqa: E402
from lensdiff_b200.types import (LensDiffEnergyMode, LensDiffFftForm, LensDiffLookMode,  # noqa: E402
                                 LensDiffSpectralMode)
from tests.helpers import OUT_TOL, rel_err, with_matrices  # noqa: E402
from tests.test_gpu_modes import _field_lens, _oracle, cache  # noqa: E402,F401

pytestmark = pytest.mark.gpu


def _render_st(cache, p, src):
    import numpy as np
    from lensdiff_b200.backend import image_request
    stream = torch.cuda.Stream()
    s = torch.from_numpy(np.ascontiguousarray(src, np.float32)).cuda()
    d = torch.full(src.shape, -7.0, device="cuda", dtype=torch.float32)
    st = cache.render(image_request(s, d, stream, frame_short_side=p.frameShortSidePx), p)
    torch.cuda.synchronize()
    assert st.ok, st
    assert cache.check_device_errors() == 0
    return d.cpu().numpy(), st


@pytest.mark.parametrize("kw", [
    {"spectralMode": LensDiffSpectralMode.Spectral5, "energyMode": LensDiffEnergyMode.Preserve,
     "fftForm": LensDiffFftForm.OwnChosen},
    {"lookMode": LensDiffLookMode.Split, "coreGain": 0.8, "structureGain": 1.2},
    {"spectralMode": LensDiffSpectralMode.Mono},
])
def test_tiled_zones_match_oracle(cache, kw):
    n = 6
    p = _field_lens(fieldGrid=n, pupilResolution=96, maxKernelRadiusPx=S.radius_percent(30, 270), **kw)
    p = p.copy(frameShortSidePx=270)
    src = S.make_frame(480, 270, 40, 1.0, 120.0, seed=81)
    out, st = _render_st(cache, with_matrices(p), src)
    Kmax = 2 * 30 + 1
    assert st.grid_used[0] < 480 + Kmax - 1 and st.grid_used[1] < 270 + Kmax - 1  # the tile grid
    orc = _oracle(p.copy(fftForm=LensDiffFftForm.OwnFp32), src, field_grid=n)
    assert rel_err(out, orc, orc[..., :3].max()) < OUT_TOL
