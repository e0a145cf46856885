"""Builds liblensdiff_b200.so in place for sm_100a.

    python -m lensdiff_b200.build [--force]

Each .cu file compiles in its own nvcc process (in parallel), then one link
step produces the shared library next to this file, where lensdiff_b200.abi
loads it.  Objects go to lensdiff_b200/_build/ (git-ignored).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "liblensdiff_b200.so")
ROOT = os.path.dirname(HERE)
SOURCES = ["ld_host.cu", "ld_psf.cu", "ld_frame.cu", "ld_frame_fx.cu", "ld_noalloc.cu", "ld_cufft.cu",
           "ld_server.cu", "ld_dftgemm.cu", "ld_debug.cu", "ld_selftest.cu"]
# cuFFT backs only the comparator form (fft_form LD_FFT_CUFFT)
LIBS = ["-L/usr/local/cuda/lib64", "-lcufft", "-Xlinker", "-rpath", "-Xlinker", "/usr/local/cuda/lib64"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", f"-I{os.path.join(ROOT, 'include')}"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _deps() -> list:
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    files.append(os.path.join(ROOT, "include", "lensdiff_b200.h"))
    files.append(os.path.abspath(__file__))
    return files


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(f) <= t for f in _deps())


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    cmd = [_nvcc(), *ARCH, *FLAGS, "-c", "-o", obj, os.path.join(CSRC, src)]
    if verbose:
        cmd.append("-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stderr[-4000:]}")
    if verbose:
        sys.stderr.write(res.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUT
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    tmp = OUT + ".tmp"
    cmd = [_nvcc(), *ARCH, "-shared", "-o", tmp, *objs, *LIBS]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stderr[-4000:]}")
    os.replace(tmp, OUT)
    return OUT


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    args = ap.parse_args()
    print(build(force=args.force, verbose=args.verbose))


if __name__ == "__main__":
    main()
