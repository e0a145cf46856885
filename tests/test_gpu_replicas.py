"""Kernel spectra handed from one library context to another (one GPU).

On a multi-GPU node one rank builds a new lens's kernel spectra and the
others take them by NCCL broadcast instead of rebuilding
(lensdiff_b200.replicas).  Here two contexts on one GPU stand for two ranks:
the block exported by one and imported by the other must give the second a
warm render (no bank or spectra rebuild) whose output equals the first's bit
for bit.  The broadcast itself runs in a one-rank NCCL group.
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from lensdiff_b200 import abi  # noqa: E402
from lensdiff_b200 import replicas as RP  # noqa: E402
from lensdiff_b200 import synthetic as S  # noqa: E402
from lensdiff_b200.backend import LensDiffPsfBankCache, image_request  # noqa: E402
from lensdiff_b200.types import LensDiffFftForm  # noqa: E402

pytestmark = pytest.mark.gpu


def _workload():
    p, _ = S.workload_hd()
    frame = S.make_frame(1920, 1080, 64, 1.0, 200.0, seed=91)
    return p.copy(fftForm=LensDiffFftForm.OwnChosen), frame


def _render(c, p, frame, stream):
    src = torch.from_numpy(frame).cuda()
    dst = torch.full_like(src, -7.0)
    st = c.render(image_request(src, dst, stream, frame_short_side=p.frameShortSidePx), p)
    stream.synchronize()
    assert st.ok, st
    return st, dst.cpu().numpy()


def test_spectra_export_import_gives_an_identical_warm_render():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    p, frame = _workload()
    H, W = frame.shape[:2]
    stream = torch.cuda.Stream()
    a, b = LensDiffPsfBankCache(0), LensDiffPsfBankCache(0)
    try:
        st_a, out_a = _render(a, p, frame, stream)
        assert st_a.bank_rebuilt and st_a.spectra_rebuilt
        nbytes, st = a.kernel_spectra_bytes(p, W, H)
        assert st.ok and nbytes > 0
        block = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        st = a.export_kernel_spectra(p, W, H, block, stream)
        assert st.ok and not st.spectra_rebuilt  # a held them already
        st = b.import_kernel_spectra(p, W, H, block, nbytes, stream)
        assert st.ok, st
        st_b, out_b = _render(b, p, frame, stream)
        assert not st_b.bank_rebuilt and not st_b.spectra_rebuilt
        assert np.array_equal(out_a, out_b)
        assert a.check_device_errors() == 0 and b.check_device_errors() == 0
    finally:
        a.close()
        b.close()


def test_spectra_transfer_refusals():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    p, frame = _workload()
    H, W = frame.shape[:2]
    stream = torch.cuda.Stream()
    c = LensDiffPsfBankCache(0)
    try:
        nbytes, _ = c.kernel_spectra_bytes(p, W, H)
        small = torch.empty(16, dtype=torch.uint8, device="cuda")
        st = c.export_kernel_spectra(p, W, H, small, stream)
        assert st.code == abi.LD_ERR_ARG and st.stage == "spectra-buffer-too-small"
        st = c.import_kernel_spectra(p, W, H, small, 16, stream)
        assert st.code == abi.LD_ERR_ARG and st.stage == "spectra-size-mismatch"
        zones = p.copy(phaseFieldStrength=1.0, phaseFieldComaRadial=0.2)
        _, st = c.kernel_spectra_bytes(zones, W, H)
        assert st.code == abi.LD_ERR_UNSUPPORTED
    finally:
        c.close()


def test_share_kernel_spectra_in_a_one_rank_nccl_group():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import torch.distributed as dist

    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ.setdefault("MASTER_PORT", "29531")
    p, frame = _workload()
    H, W = frame.shape[:2]
    stream = torch.cuda.Stream()
    dist.init_process_group("nccl", rank=0, world_size=1)
    c = LensDiffPsfBankCache(0)
    try:
        info = RP.share_kernel_spectra(c, p, W, H, stream)
        assert info["decision"] in ("broadcast", "rebuild")
        assert info["rebuild_ms"] > 0.0 and info["bytes"] > 0
        st, _ = _render(c, p, frame, stream)
        assert not st.spectra_rebuilt  # the source rank built them
    finally:
        c.close()
        dist.destroy_process_group()
