"""Serving with continuous batching (ld_server_*): frames submitted together
overlap on the GPU in separate slots, and each result is the same as when the
frame is rendered alone, within the output tolerance (2e-4 of the frame max).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from lensdiff_b200 import abi  # noqa: E402
from lensdiff_b200 import synthetic as S  # noqa: E402
from lensdiff_b200.serving import LensDiffServer  # noqa: E402
from lensdiff_b200.types import (LensDiffApertureMode, LensDiffEnergyMode,  # noqa: E402
                                 LensDiffSpectralMode)
from oracle import ref_lib as R  # noqa: E402
from tests.helpers import OUT_TOL, rel_err, with_matrices  # noqa: E402

pytestmark = pytest.mark.gpu


def _jobs():
    def lens(short, **kw):
        p = S.base_params(short)
        p.apertureMode = LensDiffApertureMode.Polygon
        p.pupilResolution = 128
        p.phaseDefocus = 0.2
        p.maxKernelRadiusPx = S.radius_percent(25, short)
        p.diffractionScalePx = 3.0
        for k, v in kw.items():
            setattr(p, k, v)
        return with_matrices(p)

    a = (S.make_frame(256, 144, 20, 1.0, 80.0, seed=21),
         lens(144, spectralMode=LensDiffSpectralMode.Tristimulus, bladeCount=6))
    b = (S.make_frame(320, 180, 24, 1.0, 60.0, seed=22),
         lens(180, spectralMode=LensDiffSpectralMode.Spectral5, bladeCount=9, roundness=0.4))
    c = (S.make_frame(200, 120, 12, 1.0, 50.0, seed=23),
         lens(120, spectralMode=LensDiffSpectralMode.Mono, energyMode=LensDiffEnergyMode.Preserve))
    return [a, b, c]


@pytest.fixture(scope="module")
def gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _alone(srv, jobs):
    out = []
    for src, p in jobs:
        t, dst = srv.submit(src, p)
        st, _ = srv.wait(t)
        assert st.ok, st
        out.append(dst.copy())
    return out


def test_results_same_alone_and_in_the_mix(gpu):
    jobs = _jobs()
    srv = LensDiffServer(0, slots=3)
    try:
        alone = _alone(srv, jobs)
        srv.reset_stats()
        order = [0, 1, 2, 0, 1, 2, 1, 0]
        tickets = [(i,) + srv.submit(jobs[i][0], jobs[i][1]) for i in order]
        for i, t, dst in tickets:
            st, lat = srv.wait(t)
            assert st.ok, st
            assert lat > 0.0
            assert rel_err(dst, alone[i], alone[i][..., :3].max()) < OUT_TOL
        stats = srv.stats()
        assert stats["completed"] == len(order)
        assert stats["max_concurrent"] >= 2  # frames overlapped on the device
        assert stats["cache_hits"] >= 3      # repeated lenses found their slot's bank
        assert 0.0 < stats["p50_ms"] <= stats["p99_ms"]
    finally:
        srv.close()
    # the served frame is the reference's frame
    if R.available():
        src, p = jobs[0]
        ref = R.render(p.copy(frameShortSidePx=144), src)
        assert rel_err(alone[0], ref, ref[..., :3].max()) < OUT_TOL


def test_hbm_budget_admits_one_frame_at_a_time(gpu):
    jobs = _jobs()
    lib = abi.lib()
    ests = [lib.ld_estimate_device_bytes(abi.to_abi_params(p.copy(frameShortSidePx=min(src.shape[:2]))),
                                         src.shape[1], src.shape[0]) for src, p in jobs]
    # room for the largest frame, never for two
    srv = LensDiffServer(0, slots=3, hbm_budget_bytes=int(max(ests) + 0.5 * min(ests)))
    try:
        alone = _alone(srv, jobs)
        srv.reset_stats()
        tickets = [(i,) + srv.submit(jobs[i][0], jobs[i][1]) for i in (2, 1, 0, 2)]
        for i, t, dst in tickets:
            st, _ = srv.wait(t)
            assert st.ok, st
            assert rel_err(dst, alone[i], alone[i][..., :3].max()) < OUT_TOL
        assert srv.stats()["max_concurrent"] == 1
    finally:
        srv.close()


def test_frame_larger_than_the_budget_is_refused(gpu):
    src, p = _jobs()[0]
    srv = LensDiffServer(0, slots=2, hbm_budget_bytes=1 << 20)
    try:
        t, _ = srv.submit(src, p)
        st, _ = srv.wait(t)
        assert st.code == abi.LD_ERR_BUDGET and "budget" in st.stage
    finally:
        srv.close()
