"""Replicas on several GPUs of one node: one process per GPU renders its own
frames (the path does not shard inside a frame), and a new lens's kernel
spectra are either built by one rank and broadcast to the others over NVLink
(NCCL broadcast of one device block, no multicast loads) or rebuilt by every
rank, whichever costs less by measurement.

The decision compares the source rank's measured rebuild time (CUDA events
around the build) with the transfer estimate bytes / link bandwidth + a fixed
latency; every rank takes the same decision from the same broadcast numbers,
so every rank issues the same collectives in the same order.

`share_protocol` is the transport-independent protocol (tested on CPU ranks
over gloo); `share_kernel_spectra` runs it on a LensDiffPsfBankCache with
device buffers and the process group's backend (NCCL on GPUs).
"""
from __future__ import annotations

import math
from typing import Callable, Dict, Optional

# measured NVLink peer copy, GB/s per direction (a B200 node of this pool)
NVLINK_GBS = 770.0
# fixed cost of one broadcast launch, ms
BROADCAST_LATENCY_MS = 0.05


def transfer_ms(nbytes: int, link_gbs: float = NVLINK_GBS, latency_ms: float = BROADCAST_LATENCY_MS) -> float:
    return latency_ms + nbytes / (link_gbs * 1e9) * 1e3


def choose_transfer(rebuild_ms: float, nbytes: int, link_gbs: float = NVLINK_GBS,
                    latency_ms: float = BROADCAST_LATENCY_MS) -> str:
    """'broadcast' when sending the block is cheaper than rebuilding it, else 'rebuild'.
    An unknown rebuild time (nan or inf: the source held the block already) broadcasts."""
    if not math.isfinite(rebuild_ms):
        return "broadcast"
    return "broadcast" if transfer_ms(nbytes, link_gbs, latency_ms) < rebuild_ms else "rebuild"


def share_protocol(dist, group, rank: int, src_rank: int, nbytes: int,
                   build_on_source: Callable[[], "tuple"],
                   install: Callable[[object], None],
                   build_local: Callable[[], None],
                   empty_block: Callable[[int], object],
                   scalar: Callable[[float], object],
                   link_gbs: float = NVLINK_GBS, latency_ms: float = BROADCAST_LATENCY_MS) -> Dict:
    """One lens's kernel spectra across the ranks of `group`.

    build_on_source() -> (block, rebuild_ms) runs on src_rank only; install(block)
    puts a received block into a non-source rank's cache; build_local() builds
    it there instead; empty_block(n) / scalar(v) make the tensors the
    collectives carry (device tensors for NCCL, CPU tensors for gloo)."""
    block = None
    t = scalar(float("nan"))
    if rank == src_rank:
        block, rebuild_ms = build_on_source()
        t.fill_(float(rebuild_ms))
    dist.broadcast(t, src_rank, group=group)
    rebuild_ms = float(t.item())
    decision = choose_transfer(rebuild_ms, nbytes, link_gbs, latency_ms)
    if decision == "broadcast":
        if rank != src_rank:
            block = empty_block(nbytes)
        dist.broadcast(block, src_rank, group=group)
        if rank != src_rank:
            install(block)
    elif rank != src_rank:
        build_local()
    return {"decision": decision, "rebuild_ms": rebuild_ms, "transfer_ms": transfer_ms(nbytes, link_gbs, latency_ms),
            "bytes": nbytes}


def share_kernel_spectra(cache, params, width: int, height: int, stream, group=None, src_rank: int = 0,
                         link_gbs: float = NVLINK_GBS, latency_ms: float = BROADCAST_LATENCY_MS) -> Dict:
    """share_protocol on a LensDiffPsfBankCache: the source rank builds (or
    finds) the lens's kernel spectra for a width x height frame and either
    broadcasts them or lets every rank rebuild; afterwards every rank's next
    render of that lens and size starts from cached spectra."""
    import torch
    import torch.distributed as dist

    rank = dist.get_rank(group)
    dev = torch.device("cuda", torch.cuda.current_device())
    nbytes, st = cache.kernel_spectra_bytes(params, width, height)
    if not st.ok:
        raise RuntimeError(f"kernel spectra size: {st}")
    on_gpu = dist.get_backend(group) == "nccl"
    tdev = dev if on_gpu else torch.device("cpu")

    def build_on_source():
        buf = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s = cache.export_kernel_spectra(params, width, height, buf, stream)
        e1.record(stream)
        e1.synchronize()
        if not s.ok:
            raise RuntimeError(f"kernel spectra export: {s}")
        ms = e0.elapsed_time(e1) if (s.spectra_rebuilt or s.bank_rebuilt) else float("inf")
        return (buf if on_gpu else buf.cpu()), ms

    def install(block):
        b = block if on_gpu else block.to(dev)
        s = cache.import_kernel_spectra(params, width, height, b, nbytes, stream)
        if not s.ok:
            raise RuntimeError(f"kernel spectra import: {s}")
        stream.synchronize()

    def build_local():  # the export builds what the context lacks; its copy is dropped
        scratch = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        s = cache.export_kernel_spectra(params, width, height, scratch, stream)
        if not s.ok:
            raise RuntimeError(f"kernel spectra rebuild: {s}")
        stream.synchronize()

    return share_protocol(dist, group, rank, src_rank, nbytes, build_on_source, install, build_local,
                          lambda n: torch.empty(n, dtype=torch.uint8, device=tdev),
                          lambda v: torch.tensor([v], dtype=torch.float64, device=tdev),
                          link_gbs, latency_ms)


def max_over_ranks(value: float, dist=None, group=None, device: Optional[object] = None) -> float:
    """The largest of every rank's value (a device time: the job ends with the slowest rank)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def replica_seed(base: int, rank: int) -> int:
    """Each rank renders its own frames: the workload generator's seed per rank."""
    return int(base) + int(rank)


def job_throughput(world_size: int, steps: int, max_ms: float) -> float:
    """Frames per second of the whole job: every rank's frames over the slowest rank's time."""
    return world_size * steps / (max_ms / 1000.0)
