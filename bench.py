"""Benchmark of the LensDiff diffraction path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl own|reference]
                    [--workload uhd31|hd16|small3|zones8] [--bank cold|warm]
    python bench.py --lens-set [--lenses 256]     (PSF banks of unrelated lenses)
    python bench.py --serving                     (Poisson frame serving)

A step renders one frame of the workload through the path: with --bank cold
(the default, the headline) every frame changes the defocus coefficient by
1e-6 waves, so the 31-wavelength PSF bank and the kernel spectra are rebuilt
on every frame; --bank warm keeps them cached.  Inputs (a 3840x2160 RGBA f32
frame, ~133 MB, plus >1 GB of spectra) are larger than the 126 MB L2.

value  frames/s over the whole job: frames of all ranks / max-over-ranks
       device time (CUDA events on the rendering stream), inputs resident.
e2e    the same metric through the public entry point with host buffers:
       each step copies the frame from pinned host memory, renders, and
       copies the result back (both copies inside the timed region).

The Python garbage collector is paused inside timed regions, as timeit does:
a collection pause of this driver script would idle the GPU between frames.

Multi-GPU: the path does not shard inside a frame; each rank renders its own
frames (replicas), timing is the max over ranks.

--impl reference times the reference's own CPU implementation (built from its
sources into oracle/_ref/libldref.so) on this machine's host cores.
"""
from __future__ import annotations

import argparse
import gc
import json
import math
import multiprocessing as mp
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "uhd31": "workload_uhd31",
    "hd16": "workload_hd",
    "small3": "workload_small",
    "zones8": "workload_zones8",
}
METRIC = "UHD frames/s (31-wavelength PSF bank, FFT convolution, composite)"


FFT_FORMS = {"own": 0, "chosen": 1, "cufft": 2}
FORM_NAMES = {"own": "own_fp32", "chosen": "own_chosen", "cufft": "cufft"}
# the arithmetic each form computes in
FORM_DTYPES = {"own": "f32", "cufft": "f32",
               "chosen": ("f32 frame math; bf16x3-split psf windows (f32 accumulate); fp16 frame spectra "
                          "(row spectra scaled per row tile, kernel spectra and column outputs per column)")}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="own", choices=["own", "reference"])
    ap.add_argument("--workload", default="uhd31", choices=sorted(WORKLOADS))
    ap.add_argument("--bank", default="cold", choices=["cold", "warm"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fft-form", default="chosen", choices=sorted(FFT_FORMS),
                    help="transform chain of the headline line (own: hand-written FP32)")
    ap.add_argument("--serving", action="store_true",
                    help="Poisson stream of mixed-size frames through the continuous-batching server")
    ap.add_argument("--lens-set", action="store_true",
                    help="lens-set workload: the PSF banks of --lenses unrelated lenses per step")
    ap.add_argument("--lenses", type=int, default=256, help="lenses per step of --lens-set")
    ap.add_argument("--rates", default="5,20,50,100,200", help="arrival rates (frames/s) of --serving")
    ap.add_argument("--requests", type=int, default=48, help="requests per rate of --serving")
    ap.add_argument("--slots", type=int, default=4, help="server slots of --serving")
    ap.add_argument("--no-comparators", action="store_true",
                    help="skip timing the other transform chains on the same workload")
    ap.add_argument("--no-other-workloads", action="store_true",
                    help="skip the short runs of the 8x8-zone and lens-set workloads added to the line")
    ap.add_argument("--no-error-check", action="store_true",
                    help="skip stating each form's error against the FP64 oracle (outside the timed regions)")
    return ap.parse_args()


def gpu_local_cpus(dev):
    """The host CPUs NVML reports as local to GPU `dev` (its NUMA node), among
    those this process may run on; None when NVML cannot say.  The end-to-end
    leg runs there, so its pinned frame buffers are placed in that node's
    memory and the copies do not cross the socket interconnect."""
    try:
        import pynvml
        import torch

        pr = torch.cuda.get_device_properties(dev)
        bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
        pynvml.nvmlInit()
        try:
            h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            words = pynvml.nvmlDeviceGetCpuAffinity(h, ((os.cpu_count() or 1) + 63) // 64)
        finally:
            pynvml.nvmlShutdown()
        cpus = {64 * w + b for w, m in enumerate(words) for b in range(64) if (int(m) >> b) & 1}
        cpus &= os.sched_getaffinity(0)
        return cpus or None
    except Exception:
        return None


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ---------------------------------------------------------------------------
# reference CPU timing (oracle/_ref: the reference's own CPU code)
# ---------------------------------------------------------------------------
def _ref_unit(args):
    """One unit of the reference's per-frame work for one wavelength: one bin
    convolution of the full frame driver with a kernel of the bank's size
    (convolveScalar, LensDiffCpuReference.cpp:1167-1193) plus one raw PSF of
    the bank (buildShiftedRawPsf, :831-859).  Returns seconds."""
    w, h, k, np_, s = args
    import numpy as np

    sys.path.insert(0, ROOT)
    from oracle import ref_lib as R

    rng = np.random.default_rng(7)
    d = np.zeros((h, w), np.float32)
    d[rng.integers(0, h, 64), rng.integers(0, w, 64)] = 10.0
    ker = np.ones((k, k), np.float32) / float(k * k)
    pupil = np.ones((np_, np_), np.float32)
    t = time.perf_counter()
    R.convolve_scalar(d, ker)
    R.raw_psf_from(pupil, None, s)
    return time.perf_counter() - t


def _ref_psf_unit(args):
    """One raw PSF of the reference (buildShiftedRawPsf,
    LensDiffCpuReference.cpp:831-859): pupil np_ -> PSF size s.  Seconds."""
    np_, s = args
    import numpy as np

    sys.path.insert(0, ROOT)
    from oracle import ref_lib as R

    pupil = np.ones((np_, np_), np.float32)
    t = time.perf_counter()
    R.raw_psf_from(pupil, None, s)
    return time.perf_counter() - t


def reference_units(w, h, k, np_, s, workers):
    """Runs `workers` units in parallel (spawned processes); returns their times."""
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        return pool.map(_ref_unit, [(w, h, k, np_, s)] * workers)


def cpu_baseline(w, h, k, np_, s, bins, workers):
    times = reference_units(w, h, k, np_, s, workers)
    t = max(times)
    value = workers / (bins * t)  # frames/s: each frame needs `bins` units
    return {
        "value": value,
        "unit": "frames/s",
        "cores": workers,
        "kind": "reference",
        "sample": (f"{workers} processes x 1 unit = reference convolveScalar of the {w}x{h} driver with a "
                   f"{k}x{k} kernel + reference buildShiftedRawPsf {np_}->{s}; a frame is {bins} units "
                   f"(one per wavelength, effect kernel only); unit time {t:.2f} s"),
    }


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from lensdiff_b200 import synthetic as S
    from oracle import ref_lib as R
    from oracle import ld_oracle as O

    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libldref.so not built (reference sources absent)"}))
        return
    p, frame = getattr(S, WORKLOADS[args.workload])()
    np_, s, rmax = O.resolve_sizes(p)
    bins = len(O.wavelengths(p))
    h, w = frame.shape[:2]
    workers = os.cpu_count() or 1
    for _ in range(args.warmup):
        reference_units(w, h, 2 * rmax + 1, np_, s, 1)
    t0 = time.perf_counter()
    step_times = []
    for _ in range(args.steps):
        ts = time.perf_counter()
        reference_units(w, h, 2 * rmax + 1, np_, s, workers)
        step_times.append(time.perf_counter() - ts)
    total = time.perf_counter() - t0
    frames = args.steps * workers / bins
    value = frames / total
    ms = total * 1000.0 / args.steps
    line = {
        "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "frame": [w, h], "wavelengths": bins, "pupil": np_, "psf": s,
                   "max_kernel_radius": rmax},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "frames/s", "cores": workers, "kind": "reference",
                         "sample": (f"each step: {workers} spawned processes, each one reference bin convolution "
                                    f"({w}x{h}, kernel {2 * rmax + 1}^2) + one reference raw PSF ({np_}->{s}); "
                                    f"{bins} such units per frame")},
        "e2e": {"value": value, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# clocks sampler
# ---------------------------------------------------------------------------
class Clocks:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        # LD_CLOCKS_DIR keeps the raw samples; by default they go to the temp directory
        self.path = os.path.join(os.environ.get("LD_CLOCKS_DIR", tempfile.gettempdir()),
                                 f"clocks_bench_{os.getpid()}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sms, maxs, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sms.append(float(parts[1]))
                    maxs = max(maxs, float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        if not sms:
            return None
        sms.sort()
        return {"sm_mhz": sms[len(sms) // 2], "sm_max_mhz": maxs, "reasons": sorted(reasons),
                "samples": len(sms)}


# DRAM read + write per launch (bytes, median over the run's launches; the
# lambda-rescale's pair and single-wavelength launches of one bank summed) of the
# UHD 31-wavelength cold workload's kernels, by transform form, from one
# one-pass ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) of the
# kernel sources whose digest is TRAFFIC_SOURCES_SHA (sources_digest()).  Any
# other revision of the kernels reports traffic null: a figure measured on
# other code says nothing about this code.  Writes still resident in L2 when a
# kernel ends are not counted.
TRAFFIC_SOURCES_SHA = "d7f4cd7799c9133d"
MEASURED_TRAFFIC_UHD31 = {
    "chosen": {
        "resample": 78053376,
        "crop_sum": 40304640,
        "combine": 132500224,
        "kspec_rows": 19684864,
        "kspec_cols": 105022976,
        "frame_rows": 140078848,
        "frame_cols": 146548480,
        "frame_inverse": 291208192,
        "dft_gemm": 56408320,
    },
}


def measured_traffic(workload, bank, form):
    """The measured per-kernel DRAM bytes of `form` on this workload, or None
    when they were not measured on these kernel sources (another digest,
    another workload or bank mode)."""
    if workload != "uhd31" or bank != "cold" or sources_digest() != TRAFFIC_SOURCES_SHA:
        return None
    return MEASURED_TRAFFIC_UHD31.get(form)


def sources_digest() -> str:
    """sha256 (first 16 hex digits) of the CUDA sources of the library."""
    import hashlib

    csrc = os.path.join(ROOT, "lensdiff_b200", "csrc")
    h = hashlib.sha256()
    for name in sorted(os.listdir(csrc)):
        if name.endswith((".cu", ".cuh", ".h")):
            with open(os.path.join(csrc, name), "rb") as f:
                h.update(name.encode() + b"\0" + f.read())
    return h.hexdigest()[:16]


# ---------------------------------------------------------------------------
# algorithmic bytes per launch of the frame-chain kernels
# ---------------------------------------------------------------------------
def algorithmic_bytes(W, H, grid, n_drv, n_ker, n_out, out_pixels, B=0, K=0, h16=False):
    """Bytes each frame kernel must move with this algorithm (complex = 8 B,
    4 B for the kernel spectra, column outputs and one-driver row spectra of
    the chosen form, h16, whose row spectra also carry one exponent byte per
    row): frame_rows reads the RGBA source and writes the H x (Px/2+1) row spectra;
    frame_cols reads them and the kernel spectra (Py x (Px/2+1) each) and writes
    H x (Px/2+1) per output; frame_inverse reads those, re-reads the source for
    the composite and writes the RGBA output."""
    Px, Py = grid
    bins = Px // 2 + 1
    row_spec = (4 * H * bins + H) if (h16 and n_drv == 1) else 8 * H * bins
    cplx = 4 if h16 else 8
    out_spec = cplx * H * bins
    canvas = 4 * B * K * K
    Kp = K + (K & 1)
    return {
        # bank passes over the B canvases of K x K floats (written once by the
        # lambda-rescale, which also takes the shaping statistics; read by the
        # crop sums and the combination)
        "resample": canvas, "shape_stats": 2 * canvas, "crop_sum": canvas,
        "combine": canvas + 4 * n_ker * K * K,
        "kspec_rows": 4 * n_ker * K * K + 8 * n_ker * Kp * bins,
        "kspec_cols": 8 * n_ker * Kp * bins + cplx * n_ker * Py * bins,
        "frame_rows": 16 * W * H + n_drv * row_spec,
        "frame_cols": n_drv * row_spec + n_ker * cplx * Py * bins + n_out * out_spec,
        "frame_inverse": n_out * out_spec + 16 * W * H + 16 * out_pixels,
    }


SERVING_SIZES = [((1920, 1080), 0.4, 256), ((2048, 1080), 0.2, 256), ((3840, 2160), 0.3, 512),
                 ((6144, 3160), 0.1, 750)]  # (frame, share, kernel radius px; 4R keeps the PSF grid 5-smooth)


def _reference_matrices(p):
    """The reference's spectral matrices of p's mode (BuildLensDiffSpectrumConfig
    output committed with the golden fixtures)."""
    from lensdiff_b200.types import LensDiffSpectralMode, LensDiffSpectrumStyle

    with open(os.path.join(ROOT, "tests", "golden", "spectrum_matrices.json")) as f:
        mats = json.load(f)
    m = mats[f"{LensDiffSpectralMode(int(p.spectralMode)).name}/{LensDiffSpectrumStyle(int(p.spectrumStyle)).name}"]
    return p.copy(naturalMatrix=m["natural"], styleMatrix=m["style"])


def reference_cuda_comparator(args, cache, dev):
    """The reference's RunLensDiffCuda (source/src/cuda/LensDiffCuda.cu,
    compiled unchanged with its cuFFT transforms, oracle/_ref/libldrefcuda.so)
    and the library's chosen form, both cold (bank rebuilt every frame), on
    the UHD frame at the reference-expressible setting (Spectral9, pupil 512,
    kernel radius 512 px); device time by CUDA events around each frame, plus
    the two outputs' difference.  The reference synchronises the host inside
    each call, so its event time equals its wall time."""
    import numpy as np
    import torch
    from lensdiff_b200 import synthetic as S
    from lensdiff_b200.backend import image_request
    from oracle import ref_lib as R

    if not R.cuda_available():
        return {"reference_cuda": {"unavailable": "oracle/_ref/libldrefcuda.so not built"}}
    p, frame = S.workload_reference_uhd()
    ours = _reference_matrices(p.copy(fftForm=FFT_FORMS["chosen"]))
    H, W = frame.shape[:2]
    stream = torch.cuda.Stream(device=dev)
    src = torch.from_numpy(frame).to(dev)
    dst_ref = torch.empty_like(src)
    dst_own = torch.empty_like(src)
    req = image_request(src, dst_own, stream, frame_short_side=p.frameShortSidePx)
    n = max(3, min(args.steps, 10))

    def time_frames(fn, count):
        ms = []
        for i in range(count):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn(i)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return ms

    def ref_frame(i):
        R.cuda_render(p.copy(phaseDefocus=p.phaseDefocus + 1e-6 * (i + 1)), src.data_ptr(), dst_ref.data_ptr(), W, H,
                      stream.cuda_stream, instance=0)

    def own_frame(i):
        with torch.cuda.stream(stream):
            st = cache.render(req, ours.copy(phaseDefocus=ours.phaseDefocus + 1e-6 * (i + 1)))
        if not st.ok:
            raise RuntimeError(f"render failed: {st}")

    def ref_frame_warm(i):  # the same lens every frame: the reference's bank cache hits
        R.cuda_render(p, src.data_ptr(), dst_ref.data_ptr(), W, H, stream.cuda_stream, instance=2)

    def own_frame_warm(i):
        with torch.cuda.stream(stream):
            st = cache.render(req, ours)
        if not st.ok:
            raise RuntimeError(f"render failed: {st}")

    torch.cuda.synchronize(dev)
    time_frames(ref_frame, 2)
    ref_ms = time_frames(ref_frame, n)
    time_frames(ref_frame_warm, 2)
    ref_warm_ms = time_frames(ref_frame_warm, n)
    time_frames(own_frame, 3)
    own_ms = time_frames(own_frame, n)
    time_frames(own_frame_warm, 3)
    own_warm_ms = time_frames(own_frame_warm, n)
    # one frame of each at the unperturbed setting: how far apart they are
    R.cuda_render(p, src.data_ptr(), dst_ref.data_ptr(), W, H, stream.cuda_stream, instance=1)
    with torch.cuda.stream(stream):
        cache.render(req, ours)
    stream.synchronize()
    a, b = dst_own.cpu().numpy(), dst_ref.cpu().numpy()
    diff = float(np.abs(a.astype(np.float64) - b).max() / max(float(b[..., :3].max()), 1e-30))

    def summary(ms):
        ms = sorted(ms)
        return {"value": 1000.0 / (sum(ms) / len(ms)), "unit": "frames/s", "ms_per_step": sum(ms) / len(ms),
                "p50_ms": ms[len(ms) // 2], "frames": len(ms)}

    setting = "3840x2160 Spectral9 (reference spectral matrices), pupil 512 -> PSF 2048, kernel radius 512 px"
    return {"reference_cuda": dict(summary(ref_ms), config=setting + ", cold", warm=summary(ref_warm_ms),
                                   what="reference RunLensDiffCuda (LensDiffCuda.cu unchanged, cuFFT transforms)"),
            "own_chosen_at_reference_setting": dict(summary(own_ms), config=setting + ", cold",
                                                    warm=summary(own_warm_ms),
                                                    out_diff_vs_reference_cuda=float(f"{diff:.3e}"))}


def other_workloads(dev, form):
    """Short device-timed runs of the other measured workloads in transform
    form `form` (a FFT_FORMS key), so one default run reports them too (full
    runs: --workload zones8, --lens-set):
      zones8    the UHD 31-wavelength frame with an 8x8 grid of field zones
                (64 banks, 64 convolutions per frame), cold, 3 frames after
                2 untimed ones (the first calibrates, the second captures
                the chain's CUDA graph);
      lens_set  the banks of 256 unrelated lenses per step (pupil 128-1024,
                PSF 2-4x, 8-64 wavelengths), cold, 2 steps."""
    import torch
    from lensdiff_b200 import synthetic as S
    from lensdiff_b200.backend import LensDiffPsfBankCache, image_request

    out = {}
    stream = torch.cuda.Stream(device=dev)

    def timed(fn, warm, n):
        """Mean and median device ms per step of n steps after `warm`."""
        for i in range(warm):
            fn(i)
        torch.cuda.synchronize(dev)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(n + 1)]
        ev[0].record(stream)
        for i in range(n):
            fn(warm + i)
            ev[i + 1].record(stream)
        torch.cuda.synchronize(dev)
        per = sorted(ev[i].elapsed_time(ev[i + 1]) for i in range(n))
        return ev[0].elapsed_time(ev[-1]) / n, per[n // 2]

    p, frame = S.workload_zones8()
    p = p.copy(fftForm=FFT_FORMS[form])
    cache = LensDiffPsfBankCache(dev.index or 0)
    src = torch.from_numpy(frame).to(dev)
    dst = torch.empty_like(src)
    req = image_request(src, dst, stream, frame_short_side=p.frameShortSidePx)

    def zone_frame(i):
        with torch.cuda.stream(stream):
            st = cache.render(req, p.copy(phaseDefocus=p.phaseDefocus + 1e-6 * (i + 1)))
        if not st.ok:
            raise RuntimeError(f"zones8 render failed: {st}")

    ms, med = timed(zone_frame, 2, 3)
    out["zones8"] = {"value": 1000.0 / ms, "unit": "frames/s", "ms_per_step": ms, "median_ms": med, "bank": "cold",
                     "fft_form": FORM_NAMES[form],
                     "config": "3840x2160, 8x8 field zones (64 banks x 31 wavelengths), pupil 512 -> PSF 2048"}
    cache.close()
    lenses = [q.copy(fftForm=FFT_FORMS[form]) for q in S.lens_instances(256)]
    cache = LensDiffPsfBankCache(dev.index or 0)

    def lens_step(i):
        st = cache.build_psf_banks([q.copy(phaseDefocus=q.phaseDefocus + 1e-6 * (i + 1)) for q in lenses], stream)
        if not st.ok or st.banks_rebuilt != len(lenses):
            raise RuntimeError(f"lens-set build failed: {st}")

    ms, med = timed(lens_step, 1, 2)
    out["lens_set"] = {"value": 256 * 1000.0 / ms, "unit": "lens banks/s", "ms_per_step": ms, "median_ms": med,
                       "bank": "cold",
                       "fft_form": FORM_NAMES[form],
                       "config": "256 unrelated lenses per step: pupil 128-1024, PSF 2-4x, 8-64 wavelengths"}
    if cache.check_device_errors():
        raise RuntimeError("device error word set by the other workloads")
    cache.close()
    return out


def error_check(args, p, frame, cache, stream, dev, forms):
    """Error of one frame rendered in each of `forms` (FORM_NAMES values)
    against the FP64 oracle (oracle/check.py), with the workload's own
    parameters.  The checker runs on the host after the timed regions."""
    import torch
    from lensdiff_b200.backend import image_request
    from oracle import check as C

    ref = C.OracleResult(p, frame)
    src = torch.from_numpy(frame).to(dev)
    dst = torch.empty_like(src)
    req = image_request(src, dst, stream, frame_short_side=p.frameShortSidePx)
    by_name = {v: k for k, v in FORM_NAMES.items()}
    out = {}
    for name in forms:
        pp = p.copy(fftForm=FFT_FORMS[by_name[name]])
        with torch.cuda.stream(stream):
            st = cache.render(req, pp)
        if not st.ok:
            raise RuntimeError(f"error-check render failed: {st}")
        _, kernels, st2 = cache.export_psf_bank(pp, stream)
        if not st2.ok:
            raise RuntimeError(f"error-check bank export failed: {st2}")
        torch.cuda.synchronize(dev)
        rep = C.error_report(kernels, dst.cpu().numpy(), ref)
        out[name] = {k: (float(f"{v:.3e}") if isinstance(v, float) else v) for k, v in rep.items()}
    return out


def run_serving(args):
    """Serving workload: Poisson arrivals at each rate of a stream mixing
    1920x1080 / 2048x1080 / 3840x2160 / 6144x3160 frames (40/20/30/10 %), 31
    wavelengths; 20 % of requests switch to a new lens (blades 5-12, rounding,
    obstruction, Zernike vector) and rebuild a PSF bank, the rest hit a slot's
    device cache.  Latency is submit -> result in host memory; HBM admission
    budget 150 GB."""
    import numpy as np
    import torch

    from lensdiff_b200 import synthetic as S
    from lensdiff_b200.serving import LensDiffServer

    rng = np.random.default_rng(2005)
    frames = {}
    for (w, h), _, _ in SERVING_SIZES:
        f = torch.from_numpy(S.make_frame(w, h, max(64, w * h // 4096), 1.0, 1000.0, seed=w + h)).pin_memory()
        frames[(w, h)] = f
    base, _ = S.workload_uhd31()

    def new_lens():
        return base.copy(bladeCount=int(rng.integers(5, 13)), roundness=float(rng.uniform(0, 1)),
                         centralObstruction=float(rng.uniform(0, 0.4)),
                         phaseDefocus=float(rng.normal(0, 0.15)), phaseComaX=float(rng.normal(0, 0.15)),
                         phaseAstigmatism0=float(rng.normal(0, 0.15)), phaseSpherical=float(rng.normal(0, 0.15)))

    sizes = [sz for sz, _, _ in SERVING_SIZES]
    probs = [pr for _, pr, _ in SERVING_SIZES]
    radius = {sz: r for sz, _, r in SERVING_SIZES}
    srv = LensDiffServer(0, slots=args.slots, hbm_budget_bytes=150 * 10 ** 9)
    sweep = []
    lens = new_lens()
    # warm-up, as a server would start: every slot renders every size once,
    # largest first (each slot's buffers reach their final size before the
    # sweep); one lens per slot, submitted together so they spread over the slots
    outs = [{sz: torch.empty_like(frames[sz]).pin_memory() for sz in sizes} for _ in range(args.slots)]
    for sz in sorted(sizes, key=lambda z: -z[0] * z[1]):
        ts = []
        for k in range(args.slots):
            p = lens.copy(maxKernelRadiusPx=S.radius_percent(radius[sz], sz[1]),
                          phaseDefocus=lens.phaseDefocus + 1e-3 * k)
            ts.append(srv.submit(frames[sz].numpy(), p, outs[k][sz].numpy())[0])
        for t in ts:
            st, _ = srv.wait(t, 300.0)
            if not st.ok:
                raise RuntimeError(f"serving warm-up failed: {st}")
    pool = [{sz: torch.empty_like(frames[sz]).pin_memory() for sz in sizes} for _ in range(2 * args.slots)]
    for rate in [float(r) for r in args.rates.split(",")]:
        srv.reset_stats()
        gaps = rng.exponential(1.0 / rate, args.requests)
        tickets = []
        t0 = time.perf_counter()
        due = t0
        misses = 0
        for i in range(args.requests):
            due += gaps[i]
            if rng.uniform() < 0.2:
                lens = new_lens()
                misses += 1
            sz = sizes[int(rng.choice(len(sizes), p=probs))]
            p = lens.copy(maxKernelRadiusPx=S.radius_percent(radius[sz], sz[1]))
            now = time.perf_counter()
            if due > now:
                time.sleep(due - now)
            dst = pool[i % len(pool)][sz].numpy()  # pinned result buffers, reused round-robin
            tickets.append(srv.submit(frames[sz].numpy(), p, dst)[0])
        for t in tickets:
            st, _ = srv.wait(t, 600.0)
            if not st.ok:
                raise RuntimeError(f"served frame failed: {st}")
        s = srv.stats()
        sweep.append({"rate": rate, "frames_per_s": s["frames_per_s"], "p50_ms": s["p50_ms"],
                      "p99_ms": s["p99_ms"], "mean_ms": s["mean_ms"], "lens_changes": misses,
                      "cache_hits": s["cache_hits"], "max_concurrent": s["max_concurrent"],
                      "device_gb": s["device_bytes"] / 1e9})
    srv.close()
    best = max(sweep, key=lambda r: r["frames_per_s"])
    print(json.dumps({
        "metric": "served frames/s and p99 ms (Poisson mix of 1080p/2K/UHD/6K, 31 wavelengths)",
        "value": best["frames_per_s"], "unit": "frames/s", "n_gpus": 1, "higher_is_better": True,
        "p50_ms": best["p50_ms"], "p99_ms": best["p99_ms"], "dtype": "f32", "data": "synthetic",
        "config": {"workload": "serving", "slots": args.slots, "requests_per_rate": args.requests,
                   "sizes": [list(sz) for sz in sizes], "shares": probs, "lens_change": 0.2,
                   "hbm_budget_gb": 150},
        "sweep": sweep}))


def run_lens_set(args):
    """Lens-set workload: each step builds the PSF banks of `--lenses`
    unrelated lenses (synthetic.lens_instances: pupil 128-1024, PSF 2-4x the
    pupil, 8-64 wavelengths, 5-9 blade polygons, Noll 2..22, chromatic focus)
    through ld_build_psf_banks, whose tensor-core windows for every (lens,
    wavelength) pair come from one persistent GEMM launch per transform pass
    and scratch chunk.  Every step changes every lens's defocus by 1e-6 waves,
    so all banks are rebuilt.  Metric: lens banks/s, device time."""
    import numpy as np
    import torch

    from lensdiff_b200 import synthetic as S
    from lensdiff_b200.backend import LensDiffPsfBankCache, resolve_sizes

    lenses = S.lens_instances(args.lenses)
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    cache = LensDiffPsfBankCache(0)
    stream = torch.cuda.Stream(device=dev)
    k = [0]

    def step():
        k[0] += 1
        st = cache.build_psf_banks([q.copy(phaseDefocus=q.phaseDefocus + 1e-6 * k[0]) for q in lenses], stream)
        if not st.ok or st.banks_rebuilt != len(lenses):
            raise RuntimeError(f"lens-set build failed: {st}")
        return st

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    clocks = Clocks(0)
    clocks.start()
    time.sleep(0.3)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    launches = 0
    gc.collect()
    gc.disable()
    evs[0].record(stream)
    for i in range(args.steps):
        launches += step().kernel_launches
        evs[i + 1].record(stream)
    torch.cuda.synchronize(dev)
    gc.enable()
    clk = clocks.stop()
    per_step = sorted(evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps))
    total_ms = evs[0].elapsed_time(evs[-1])
    # stages and tensor-core work of one profiled step
    cache.set_profiling(True)
    cache.profile_collect()
    cache.tensor_flops()
    step()
    torch.cuda.synchronize(dev)
    stage = cache.profile_collect()
    flops = cache.tensor_flops()
    cache.set_profiling(False)
    if cache.check_device_errors():
        raise RuntimeError("device error word set by the lens-set builds")
    cache.close()
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 1400.0, "fallback (sustained bf16)"
    if os.path.exists(peaks_path):
        with open(peaks_path) as f:
            pk = json.load(f)
        peak = float(pk.get("bf16_tflops_sustained", pk.get("bf16_tflops")))
        peak_src = "measured (sustained bf16)"
    g_ms, g_n = stage.get("dft_gemm", (0.0, 0))
    roofline = None
    if g_n:
        achieved = flops / g_n / (g_ms / g_n / 1000.0) / 1e12
        roofline = {"bound": "tensor", "kernel": "dft_gemm", "achieved": achieved, "peak": peak,
                    "unit": "TFLOP/s", "frac": achieved / peak, "peak_source": peak_src, "traffic": None,
                    "flops_per_launch": flops / g_n, "launch_ms": g_ms / g_n, "launches": g_n,
                    "note": "bf16 MMA flops issued, the BF16x3 split's three products counted"}
    sizes = [resolve_sizes(q) for q in lenses]
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import ref_lib as R

        if R.available():
            rng = np.random.default_rng(9)
            small = [i for i, z in enumerate(sizes) if z[1] <= 2048]
            workers = min(16, os.cpu_count() or 1)
            pick = [int(i) for i in rng.choice(small, size=min(workers, len(small)), replace=False)]
            ctx = mp.get_context("spawn")
            with ctx.Pool(len(pick)) as pool:
                ts = pool.map(_ref_psf_unit, [(sizes[i][0], sizes[i][1]) for i in pick])
            cost = lambda z: z[1] * z[1] * math.log2(z[1])  # noqa: E731
            c = float(np.mean([t / cost(sizes[i]) for t, i in zip(ts, pick)]))
            est = sum(z[3] * c * cost(z) for z in sizes) / len(pick)
            cpu = {"value": len(lenses) / est, "unit": "lens banks/s", "cores": len(pick), "kind": "reference",
                   "sample": (f"{len(pick)} processes, each one reference buildShiftedRawPsf of a sampled lens "
                              f"(PSF <= 2048); seconds per raw PSF fitted as c*S^2*log2(S), summed over every "
                              f"(lens, wavelength) of the set and divided by the processes (raw PSFs only: the "
                              f"reference's resampling and shaping are not counted)")}
    print(json.dumps({
        "metric": "lens PSF banks/s (uneven pupils, PSF sizes, wavelength counts)",
        "value": args.steps * len(lenses) / (total_ms / 1000.0), "unit": "lens banks/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "p50_ms": per_step[len(per_step) // 2], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16x3 (tensor-core DFT), f32 elsewhere", "data": "synthetic",
        "config": {"workload": f"lens_set{len(lenses)}", "lenses": len(lenses),
                   "pupil": [min(z[0] for z in sizes), max(z[0] for z in sizes)],
                   "psf": [min(z[1] for z in sizes), max(z[1] for z in sizes)],
                   "wavelengths_total": sum(z[3] for z in sizes), "bank": "cold",
                   "l2": "inputs larger than L2 (tens of GB of windows and canvases per step)"},
        "gpu_launches": launches,
        "stage_ms_per_step": {k: round(v[0], 3) for k, v in stage.items() if v[1]},
        "roofline": roofline, "clocks": clk, "cpu_baseline": cpu}))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.serving:
        run_serving(args)
        return
    if args.lens_set:
        run_lens_set(args)
        return
    ws, rank, local = dist_env()
    import numpy as np
    import torch

    pool_ctx = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    else:
        torch.cuda.set_device(local)
    from lensdiff_b200 import synthetic as S
    from lensdiff_b200.backend import LensDiffPsfBankCache, image_request

    from lensdiff_b200 import replicas as RP

    p, frame = getattr(S, WORKLOADS[args.workload])(seed=RP.replica_seed(1003, rank))
    p = p.copy(fftForm=FFT_FORMS[args.fft_form])
    H, W = frame.shape[:2]
    dev = torch.device("cuda", local)
    cache = LensDiffPsfBankCache(local)
    stream = torch.cuda.Stream(device=dev)
    src = torch.from_numpy(frame).to(dev)
    dst = torch.empty_like(src)
    req = image_request(src, dst, stream, frame_short_side=p.frameShortSidePx)
    counter = [0]

    def params_for_step():
        counter[0] += 1
        if args.bank == "cold":
            return p.copy(phaseDefocus=p.phaseDefocus + 1e-6 * counter[0])
        return p

    launches_per_frame = [0]

    def step():
        st = cache.render(req, params_for_step())
        if not st.ok:
            raise RuntimeError(f"render failed: {st}")
        launches_per_frame[0] = st.kernel_launches
        return st

    with torch.cuda.stream(stream):
        st0 = step()
        for _ in range(max(0, args.warmup - 1)):
            step()
    torch.cuda.synchronize(dev)

    clocks = Clocks(local)
    clocks.start()
    time.sleep(0.3)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    gc.collect()
    gc.disable()  # a collection pause of the Python driver would idle the GPU between frames
    with torch.cuda.stream(stream):
        evs[0].record(stream)
        for i in range(args.steps):
            step()
            evs[i + 1].record(stream)
    torch.cuda.synchronize(dev)
    gc.enable()
    if ws > 1:
        torch.distributed.barrier()
    # per-stage device times from a separate profiled pass (stage events
    # bracket every launch, so the timed frames above run without them and
    # replay their per-frame chains as CUDA graphs)
    n_prof = min(args.steps, 5)
    cache.set_profiling(True)
    cache.profile_collect()
    cache.tensor_flops()  # restarts the count of tensor-core flops issued
    with torch.cuda.stream(stream):
        for _ in range(n_prof):
            step()
    torch.cuda.synchronize(dev)
    stage = cache.profile_collect()
    prof_flops = cache.tensor_flops()
    cache.set_profiling(False)
    dev_err = cache.check_device_errors()
    if dev_err:
        raise RuntimeError(f"device error word {dev_err} after the timed frames")
    clk = clocks.stop()
    per_step = [evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps)]
    sys.stderr.write("step ms: " + " ".join(f"{v:.3f}" for v in per_step) + "\n")
    total_ms = RP.max_over_ranks(evs[0].elapsed_time(evs[-1]), torch.distributed if ws > 1 else None, device=dev)
    value = RP.job_throughput(ws, args.steps, total_ms)
    ps = sorted(per_step)
    p50 = ps[len(ps) // 2]
    p99 = ps[min(len(ps) - 1, int(math.ceil(0.99 * len(ps))) - 1)]

    # ---- end to end through the public entry point with host buffers -----
    # Frames stream from pinned host memory and back: frame i+1 is copied in
    # and frame i-1 copied out while frame i renders (two device frame slots,
    # a copy-in stream, the render stream and a copy-out stream, ordered by
    # events), so the copies overlap the device work as a video host would.
    e2e = None
    if not args.no_e2e:
        all_cpus = os.sched_getaffinity(0)
        local_cpus = gpu_local_cpus(dev)
        if local_cpus:
            os.sched_setaffinity(0, local_cpus)
        host_in = torch.from_numpy(frame).pin_memory()
        host_out = [torch.empty_like(host_in).pin_memory() for _ in range(2)]
        srcs = [src, torch.empty_like(src)]
        dsts = [dst, torch.empty_like(dst)]
        reqs = [image_request(srcs[i], dsts[i], stream, frame_short_side=p.frameShortSidePx) for i in range(2)]
        s_in, s_out = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
        ev = lambda: torch.cuda.Event(enable_timing=False)  # noqa: E731
        copied_in = [ev(), ev()]
        rendered = [ev(), ev()]
        copied_out = [ev(), ev()]

        def run_frames(n):
            for i in range(n):
                j = i % 2
                with torch.cuda.stream(s_in):
                    if i >= 2:
                        s_in.wait_event(rendered[j])  # the render of frame i-2 has read srcs[j]
                    srcs[j].copy_(host_in, non_blocking=True)
                    copied_in[j].record(s_in)
                with torch.cuda.stream(stream):
                    stream.wait_event(copied_in[j])
                    if i >= 2:
                        stream.wait_event(copied_out[j])  # dsts[j] of frame i-2 is on the host
                    st = cache.render(reqs[j], params_for_step())
                    if not st.ok:
                        raise RuntimeError(f"render failed: {st}")
                    rendered[j].record(stream)
                with torch.cuda.stream(s_out):
                    s_out.wait_event(rendered[j])
                    host_out[j].copy_(dsts[j], non_blocking=True)
                    copied_out[j].record(s_out)

        run_frames(3)
        torch.cuda.synchronize(dev)
        if ws > 1:
            torch.distributed.barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        gc.collect()
        gc.disable()
        ev0.record(s_in)
        run_frames(args.steps)
        ev1.record(s_out)
        torch.cuda.synchronize(dev)
        gc.enable()
        e_ms = torch.tensor([ev0.elapsed_time(ev1)], device=dev, dtype=torch.float64)
        if ws > 1:
            torch.distributed.all_reduce(e_ms, op=torch.distributed.ReduceOp.MAX)
        nbytes = frame.nbytes
        os.sched_setaffinity(0, all_cpus)
        e2e = {"value": ws * args.steps / (float(e_ms.item()) / 1000.0), "unit": "frames/s",
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
               "pipelining": "copy-in / render / copy-out streams, two frame slots",
               "host_cpus": (f"{len(local_cpus)} local to the GPU (NVML affinity)" if local_cpus
                             else "all (no NVML affinity)")}

    # ---- roofline of the dominant kernel ----------------------------------
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        with open(peaks_path) as f:
            peak = float(json.load(f)["hbm_gbs"])
        peak_src = "measured"
    grid = st0.grid_used
    spectral = int(p.spectralMode) != 0
    n_drv = 1 if spectral else 3
    n_ker = 3 if spectral else 1
    n_out = 3
    alg = algorithmic_bytes(W, H, grid, n_drv, n_ker, n_out, W * H, h16=(args.fft_form == "chosen" and spectral),
                            B=st0.wavelength_count,
                            K=2 * st0.max_kernel_radius + 1)
    # the dominant kernel: the most device time per frame among the kernels
    # with a roofline (the HBM-bound passes; the tensor-core DFT GEMM)
    roofed = {k: v for k, v in stage.items() if v[1] and (k in alg or (k == "dft_gemm" and prof_flops > 0))}
    dominant = max(roofed or stage, key=lambda k: stage[k][0])
    dom_ms, dom_n = stage[dominant]
    roofline = None
    traffic_map = measured_traffic(args.workload, args.bank, args.fft_form)
    # every HBM-bound kernel's fraction of the measured peak (the frame chain's
    # fused FFT kernels first among them)
    kernel_frac = {}
    for name, (ms, n) in stage.items():
        if name in alg and n and ms > 0:
            kernel_frac[name] = round(alg[name] / (ms / n / 1000.0) / 1e9 / peak, 4)
    if dominant == "dft_gemm" and dom_n and prof_flops > 0:
        # tensor-bound: the MMA flops issued (the BF16x3 split's three
        # products counted) over the launch time, against the measured bf16
        # burst rate (the GEMM runs in bursts of well under a millisecond)
        tpeak, tpeak_src = 1590.0, "fallback (burst bf16)"
        if os.path.exists(peaks_path):
            with open(peaks_path) as f:
                tpeak = float(json.load(f)["bf16_tflops"])
            tpeak_src = "measured (burst bf16)"
        per_launch_ms = dom_ms / dom_n
        flops_launch = prof_flops / dom_n
        achieved = flops_launch / (per_launch_ms / 1000.0) / 1e12
        traffic = traffic_map.get(dominant) if traffic_map else None
        roofline = {"bound": "tensor", "kernel": dominant, "achieved": achieved, "peak": tpeak, "unit": "TFLOP/s",
                    "frac": achieved / tpeak, "peak_source": tpeak_src, "traffic": traffic,
                    "flops_per_launch": flops_launch, "launch_ms": per_launch_ms}
    elif dominant in alg and dom_n:
        per_launch_ms = dom_ms / dom_n
        achieved = alg[dominant] / (per_launch_ms / 1000.0) / 1e9
        traffic = traffic_map.get(dominant) if traffic_map else None
        roofline = {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "peak_source": peak_src, "traffic": traffic,
                    "algorithmic_bytes_per_launch": alg[dominant], "launch_ms": per_launch_ms}
    else:
        roofline = {"bound": "hbm", "kernel": dominant, "achieved": None, "peak": peak, "unit": "GB/s",
                    "frac": None, "peak_source": peak_src, "traffic": None}
    stage_ms = {k: round(v[0] / n_prof, 4) for k, v in stage.items() if v[1]}
    # the radix orders and launch shapes the autotuner picked for the grid
    autotune = {}
    for n in (grid[0] // 2, grid[1]):
        ch = cache.autotune_choice(n)
        if ch:
            autotune[str(n)] = {"radices": list(ch[0]), "shape": ch[1], "ms": round(ch[2], 4)}

    # ---- the same form with the bank cached (warm: the frame chain alone, as
    # a video host renders every frame after a lens change) ------------------
    warm = None
    if args.bank == "cold" and not args.no_comparators:
        wp = p.copy(phaseDefocus=p.phaseDefocus + 0.5e-6)

        def warm_step():
            st = cache.render(req, wp)
            if not st.ok:
                raise RuntimeError(f"warm render failed: {st}")

        with torch.cuda.stream(stream):
            for _ in range(max(3, args.warmup)):
                warm_step()
        torch.cuda.synchronize(dev)
        wev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
        gc.collect()
        gc.disable()
        with torch.cuda.stream(stream):
            wev[0].record(stream)
            for i in range(args.steps):
                warm_step()
                wev[i + 1].record(stream)
        torch.cuda.synchronize(dev)
        gc.enable()
        wps = sorted(wev[i].elapsed_time(wev[i + 1]) for i in range(args.steps))
        wtot = RP.max_over_ranks(wev[0].elapsed_time(wev[-1]), torch.distributed if ws > 1 else None, device=dev)
        warm = {"value": RP.job_throughput(ws, args.steps, wtot), "unit": "frames/s", "ms_per_step": wtot / args.steps,
                "p50_ms": wps[len(wps) // 2], "p99_ms": wps[min(len(wps) - 1, int(math.ceil(0.99 * len(wps))) - 1)]}

    # ---- the other transform chains on the same workload (device time) ------
    comparators = {}
    if not args.no_comparators:
        for name in ("own", "chosen", "cufft"):
            if name == args.fft_form:
                continue
            base = p.copy(fftForm=FFT_FORMS[name])
            k = [0]

            def cmp_step():
                k[0] += 1
                pp = base.copy(phaseDefocus=base.phaseDefocus + 1e-6 * (k[0] + 10000)) if args.bank == "cold" \
                    else base
                st = cache.render(req, pp)
                if not st.ok:
                    raise RuntimeError(f"{name} render failed: {st}")

            with torch.cuda.stream(stream):
                for _ in range(args.warmup):
                    cmp_step()
            torch.cuda.synchronize(dev)
            cev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
            gc.collect()
            gc.disable()
            with torch.cuda.stream(stream):
                cev[0].record(stream)
                for i in range(args.steps):
                    cmp_step()
                    cev[i + 1].record(stream)
            torch.cuda.synchronize(dev)
            gc.enable()
            cps = sorted(cev[i].elapsed_time(cev[i + 1]) for i in range(args.steps))
            ctot = torch.tensor([cev[0].elapsed_time(cev[-1])], device=dev, dtype=torch.float64)
            if ws > 1:
                torch.distributed.all_reduce(ctot, op=torch.distributed.ReduceOp.MAX)
            ctot = float(ctot.item())
            comparators[FORM_NAMES[name]] = {
                "value": ws * args.steps / (ctot / 1000.0), "unit": "frames/s", "ms_per_step": ctot / args.steps,
                "p50_ms": cps[len(cps) // 2], "p99_ms": cps[min(len(cps) - 1, int(math.ceil(0.99 * len(cps))) - 1)]}
        if cache.check_device_errors():
            raise RuntimeError("device error word set by a comparator chain")

    # ---- the reference's own CUDA chain on this GPU (1 GPU runs only) -------
    if ws == 1 and not args.no_comparators and args.workload == "uhd31":
        ref_cuda = reference_cuda_comparator(args, cache, dev)
        if ref_cuda is not None:
            comparators.update(ref_cuda)

    # ---- error against the FP64 oracle (checker only; outside every timed
    # region): one frame of the workload's own parameters in each timed form
    errors = None
    if rank == 0 and not args.no_error_check:
        forms = [n for n in comparators if n in FORM_NAMES.values()] + [FORM_NAMES[args.fft_form]]
        errors = error_check(args, p, frame, cache, stream, dev, forms)

    workloads = None
    if rank == 0 and ws == 1 and args.workload == "uhd31" and not args.no_other_workloads:
        workloads = other_workloads(dev, args.fft_form)

    # ---- CPU baseline (rank 0, N=1) ----------------------------------------
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        from oracle import ref_lib as R

        if R.available():
            cpu = cpu_baseline(W, H, 2 * st0.max_kernel_radius + 1, st0.pupil_size, st0.raw_psf_size,
                               st0.wavelength_count, os.cpu_count() or 1)
        else:
            cpu = {"value": None, "unit": "frames/s", "cores": 0, "kind": "reference",
                   "sample": "oracle/_ref/libldref.so not built"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "p50_ms": p50, "p99_ms": p99,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": FORM_DTYPES[args.fft_form],
            "data": "synthetic (seeded generator; no public dataset exists)",
            "config": {"workload": args.workload, "frame": [W, H], "wavelengths": st0.wavelength_count,
                       "pupil": st0.pupil_size, "psf": st0.raw_psf_size,
                       "max_kernel_radius": st0.max_kernel_radius, "bank": args.bank,
                       "grid_requested": list(st0.grid_requested), "grid_used": list(st0.grid_used),
                       "fft_form": FORM_NAMES[args.fft_form], "parallelism": f"replicas x{ws}",
                       "l2": "inputs larger than L2 (frame 133 MB + spectra > 1 GB)"},
            "gpu_launches": launches_per_frame[0] * args.steps,
            "stage_ms_per_frame": stage_ms,
            "roofline": roofline,
            "kernel_hbm_frac": kernel_frac,
            # DRAM bytes per launch measured on these kernel sources, beside
            # the algorithmic bytes (null on any other revision)
            "kernel_traffic": ({k: {"dram_bytes": v, "algorithmic_bytes": alg.get(k)} for k, v in traffic_map.items()}
                               if traffic_map else None),
            "autotune": autotune,
            "error": errors.get(FORM_NAMES[args.fft_form]) if errors else None,
            "clocks": clk,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "warm": warm,
            "comparators": comparators,
            "workloads": workloads,
        }
        if errors:
            for name, c in comparators.items():
                c["error"] = errors.get(name)
        print(json.dumps(line))
    cache.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
