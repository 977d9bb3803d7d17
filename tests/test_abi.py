"""The C-ABI library loads on a machine without a GPU, exports every symbol
include/rav2d_gpu.h declares, and agrees with the Python mirrors on struct
layout and plane geometry (host-only calls, no compute)."""
import ctypes as C
import os
import re

import pytest

from rav2d_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    hdr = open(os.path.join(ROOT, "include", "rav2d_gpu.h")).read()
    return sorted(set(re.findall(r"\b(r2g_\w+)\s*\(", hdr)))


@pytest.fixture(scope="module")
def lib():
    from rav2d_b200 import gpu

    return gpu.lib()


def test_exports_every_declared_symbol(lib):
    names = _declared()
    assert len(names) >= 16
    for n in names:
        assert hasattr(lib, n), n


def test_struct_sizes_match_python_mirrors(lib):
    sizes = (C.c_int32 * 16)()
    n = lib.r2g_struct_sizes(sizes, 16)
    assert n == len(abi.STRUCT_SIZES)
    for i, (name, sz) in enumerate(abi.STRUCT_SIZES):
        assert sizes[i] == sz, name


@pytest.mark.parametrize("w,h,bd", [(352, 288, 8), (1920, 1080, 10), (3840, 2160, 10), (1024, 64, 8), (512, 64, 10)])
def test_plane_geometry(lib, w, h, bd):
    vals = [C.c_int64() for _ in range(4)]
    assert lib.r2g_plane_geometry(w, h, bd, *[C.byref(v) for v in vals]) == 0
    assert tuple(v.value for v in vals) == abi.plane_geometry(w, h, bd)


def test_plane_geometry_rejects_bad_bitdepth(lib):
    v = C.c_int64()
    assert lib.r2g_plane_geometry(64, 64, 12, C.byref(v), C.byref(v), C.byref(v), C.byref(v)) == abi.R2G_E_INVALID


def test_version(lib):
    assert lib.r2g_version() >= 1
