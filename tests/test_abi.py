"""C-ABI checks that need no GPU: the library loads, exports every entry point
include/lensdiff_b200.h declares, and the ctypes mirrors have the C layout."""
import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from lensdiff_b200 import abi
from lensdiff_b200.backend import resolve_sizes
from lensdiff_b200 import synthetic as S
from oracle import ld_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "lensdiff_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|size_t)\s+(ld_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = abi.lib()
    names = declared_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(abi.EXPORTED_SYMBOLS) == names


def _c_layout():
    src = r"""
#include <stdio.h>
#include <stddef.h>
#include "lensdiff_b200.h"
#define O(T, f) printf(#T "." #f " %zu\n", offsetof(T, f))
int main(void) {
  printf("ld_params %zu\nld_render_request %zu\nld_status %zu\nld_image_view %zu\n",
         sizeof(ld_params), sizeof(ld_render_request), sizeof(ld_status), sizeof(ld_image_view));
  O(ld_params, threshold); O(ld_params, blade_count); O(ld_params, max_kernel_radius_px);
  O(ld_params, phase_defocus); O(ld_params, spectrum_force); O(ld_params, structure_shoulder);
  O(ld_params, wavelength_count); O(ld_params, natural_matrix); O(ld_params, noll); O(ld_params, fft_form);
  O(ld_render_request, src); O(ld_render_request, dst); O(ld_render_request, cuda_stream);
  O(ld_status, bank_rebuilt); O(ld_status, kernel_launches);
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    return dict(line.split() for line in out.strip().splitlines())


def test_struct_layouts_match_c():
    lay = _c_layout()
    assert int(lay["ld_params"]) == ctypes.sizeof(abi.ld_params)
    assert int(lay["ld_render_request"]) == ctypes.sizeof(abi.ld_render_request)
    assert int(lay["ld_status"]) == ctypes.sizeof(abi.ld_status)
    assert int(lay["ld_image_view"]) == ctypes.sizeof(abi.ld_image_view)
    for key, off in lay.items():
        if "." not in key:
            continue
        t, f = key.split(".")
        assert getattr(getattr(abi, t), f).offset == int(off), key


@pytest.mark.parametrize("wl", [S.workload_small, S.workload_hd, S.workload_uhd31])
def test_resolve_sizes_matches_oracle(wl):
    p, _ = wl()
    np_, s, r, b = resolve_sizes(p)
    assert (np_, s, r) == O.resolve_sizes(p)
    assert b == len(O.wavelengths(p))


def test_gaussian_rgb_matrix_matches_oracle():
    wl = np.linspace(400, 700, 31).astype(np.float32)
    out = np.zeros(3 * 31, np.float32)
    c = np.array([600, 540, 450], np.float32)
    rc = abi.lib().ld_gaussian_rgb_matrix(wl.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), 31,
                                          c.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), 40.0,
                                          out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    assert rc == 0
    ref = O.gaussian_rgb_matrix(wl, c, 40.0)
    assert np.abs(out.reshape(3, 31) - ref).max() < 1e-6
    assert np.allclose(out.reshape(3, 31).sum(axis=1), 1.0, atol=1e-5)
