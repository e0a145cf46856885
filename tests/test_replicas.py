"""The multi-GPU replica harness on two CPU ranks over gloo (no GPU).

Covers what bench.py's --gpus N run and lensdiff_b200.replicas do across
ranks: per-rank workload seeds, the max-over-ranks device time and the
whole-job throughput, and the kernel-spectra handoff protocol (the source
rank broadcasts its block when that is cheaper than a rebuild, else every
rank rebuilds), with both decisions taken identically on every rank.
"""
import os
import socket
import tempfile

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as tmp  # noqa: E402

from lensdiff_b200 import replicas as RP  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir, rebuild_ms_src, nbytes):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = {}
        # ---- replica timing: every rank's own time, the job's is the slowest
        local_ms = 10.0 + 5.0 * rank
        res["max_ms"] = RP.max_over_ranks(local_ms, dist)
        res["seed"] = RP.replica_seed(1003, rank)
        res["throughput"] = RP.job_throughput(world, 20, res["max_ms"])
        # ---- kernel-spectra handoff with a fake cache
        src_block = torch.from_numpy(np.random.default_rng(11).integers(0, 256, nbytes, dtype=np.uint8))
        installed, rebuilt = [], []

        def build_on_source():
            return src_block.clone(), rebuild_ms_src

        info = RP.share_protocol(
            dist, None, rank, 0, nbytes, build_on_source,
            install=lambda b: installed.append(b.clone()),
            build_local=lambda: rebuilt.append(True),
            empty_block=lambda n: torch.zeros(n, dtype=torch.uint8),
            scalar=lambda v: torch.tensor([v], dtype=torch.float64))
        res["decision"] = info["decision"]
        res["rebuild_ms"] = info["rebuild_ms"]
        res["installed_equal"] = bool(installed) and bool(torch.equal(installed[0], src_block))
        res["installed"] = len(installed)
        res["rebuilt"] = len(rebuilt)
        torch.save(res, os.path.join(out_dir, f"r{rank}.pt"))
    finally:
        dist.destroy_process_group()


def _run(rebuild_ms_src, nbytes):
    with tempfile.TemporaryDirectory() as d:
        tmp.spawn(_worker, args=(2, _free_port(), d, rebuild_ms_src, nbytes), nprocs=2, join=True)
        return [torch.load(os.path.join(d, f"r{r}.pt")) for r in range(2)]


def test_replica_timing_is_the_slowest_rank_and_seeds_differ():
    r0, r1 = _run(1.0, 4096)
    assert r0["max_ms"] == r1["max_ms"] == 15.0
    assert r0["throughput"] == r1["throughput"] == pytest.approx(2 * 20 / 0.015)
    assert r0["seed"] != r1["seed"]


def test_handoff_broadcasts_when_the_rebuild_costs_more():
    # 96 MB at 770 GB/s is ~0.17 ms against a 0.85 ms rebuild: broadcast
    nbytes = 1 << 20
    r0, r1 = _run(0.85, nbytes)
    assert r0["decision"] == r1["decision"] == "broadcast"
    assert r1["installed"] == 1 and r1["installed_equal"] and r1["rebuilt"] == 0
    assert r0["installed"] == 0 and r0["rebuilt"] == 0


def test_handoff_rebuilds_when_that_is_cheaper():
    r0, r1 = _run(0.01, 1 << 20)  # a 10 us rebuild beats any transfer
    assert r0["decision"] == r1["decision"] == "rebuild"
    assert r1["rebuilt"] == 1 and r1["installed"] == 0
    assert r0["rebuilt"] == 0


def test_choose_transfer_costs():
    assert RP.choose_transfer(float("inf"), 10 ** 9) == "broadcast"
    assert RP.choose_transfer(0.85, 96 * 10 ** 6) == "broadcast"   # 0.175 ms transfer
    assert RP.choose_transfer(0.1, 96 * 10 ** 6) == "rebuild"
    assert RP.transfer_ms(770 * 10 ** 6) == pytest.approx(1.0 + RP.BROADCAST_LATENCY_MS)
