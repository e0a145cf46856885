"""The benchmark's accounting, without a GPU: algorithmic bytes per frame
kernel, the gate that reports measured DRAM traffic only for the kernel
sources it was captured on, and the host-CPU placement helper."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

UHD = dict(W=3840, H=2160, grid=(5000, 3200), n_drv=1, n_ker=3, n_out=3, out_pixels=3840 * 2160)


def test_chosen_form_halves_the_spectra_bytes():
    f32 = bench.algorithmic_bytes(**UHD)
    h16 = bench.algorithmic_bytes(**UHD, h16=True)
    bins = 2501
    # row spectra: 8 bytes per value in FP32; 4 per value plus one exponent byte per row in FP16
    assert f32["frame_rows"] - h16["frame_rows"] == 8 * 2160 * bins - (4 * 2160 * bins + 2160)
    # the column pass reads row and kernel spectra and writes three column outputs, all halved
    assert h16["frame_cols"] == 4 * 2160 * bins + 2160 + 3 * 4 * 3200 * bins + 3 * 4 * 2160 * bins
    assert h16["frame_inverse"] == 3 * 4 * 2160 * bins + 2 * 16 * 3840 * 2160
    # the Mono chain (three drivers) keeps FP32 row spectra
    mono = bench.algorithmic_bytes(**dict(UHD, n_drv=3, n_ker=1), h16=True)
    assert mono["frame_rows"] == 16 * 3840 * 2160 + 3 * 8 * 2160 * bins


def test_traffic_is_reported_only_for_the_sources_it_was_measured_on(monkeypatch):
    digest = bench.sources_digest()
    assert len(digest) == 16 and int(digest, 16) >= 0
    monkeypatch.setattr(bench, "TRAFFIC_SOURCES_SHA", digest)
    monkeypatch.setattr(bench, "MEASURED_TRAFFIC_UHD31", {"chosen": {"frame_cols": 123}})
    assert bench.measured_traffic("uhd31", "cold", "chosen") == {"frame_cols": 123}
    assert bench.measured_traffic("uhd31", "cold", "own") is None
    assert bench.measured_traffic("hd16", "cold", "chosen") is None
    assert bench.measured_traffic("uhd31", "warm", "chosen") is None
    monkeypatch.setattr(bench, "TRAFFIC_SOURCES_SHA", "0" * 16)
    assert bench.measured_traffic("uhd31", "cold", "chosen") is None


def test_committed_traffic_covers_frame_kernels():
    for form, table in bench.MEASURED_TRAFFIC_UHD31.items():
        assert form in bench.FFT_FORMS
        for name in ("frame_rows", "frame_cols", "frame_inverse"):
            assert table[name] > 0


def test_gpu_local_cpus_without_a_gpu_is_none_or_a_subset():
    cpus = bench.gpu_local_cpus(0)
    assert cpus is None or cpus <= os.sched_getaffinity(0)
