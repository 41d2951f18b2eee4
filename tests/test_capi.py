"""The C-ABI library loads and exports every entry point include/tsp_b200.h declares (no GPU)."""
import ctypes as C
import os
import re

import pytest

from turbospharticles_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_entry_points():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            text = open(os.path.join(ROOT, "include", h)).read()
            names += re.findall(r"^\s*(?:int|const char\*|uint64_t)\s+(tsp_b200_\w+)\s*\(", text, re.M)
    return names


def test_header_declares_entry_points():
    names = declared_entry_points()
    assert "tsp_b200_step" in names and "tsp_b200_pull_state" in names
    assert len(names) == len(set(names))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(abi.LIB_PATH):
        from turbospharticles_b200 import build
        build.build()
    return C.CDLL(abi.LIB_PATH)


def test_library_exports_every_declared_symbol(lib):
    for name in declared_entry_points():
        assert hasattr(lib, name), name


def test_python_signatures_cover_header():
    assert set(declared_entry_points()) <= set(abi.EXPORTS)


def test_struct_layouts_match_header():
    # tsp_params: 25 four-byte fields + 4 reserved words
    assert C.sizeof(abi.TspParams) == 4 * (3 + 2 + 3 + 2 + 3 + 4 + 4 + 1 + 1 + 1 + 4)
    # tsp_state_view: 4 counts, step, time, then only pointers
    n_ptr = len(abi.TspStateView._fields_) - 6
    assert C.sizeof(abi.TspStateView) == 16 + 8 + 8 + 8 * n_ptr


def test_null_handle_is_rejected_without_gpu(lib):
    lib.tsp_b200_step.restype = C.c_int
    lib.tsp_b200_step.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
    assert lib.tsp_b200_step(None, None, 1) == -1
    lib.tsp_b200_last_error.restype = C.c_char_p
    lib.tsp_b200_last_error.argtypes = [C.c_void_p]
    assert b"NULL" in lib.tsp_b200_last_error(None)


# ---- cell frame rule (tests/unit/cell_frame.cpp of the reference, through the C ABI)
def _frame(lib_abi, lo, hi, orig=(4, 5, 6), dims=(7, 8, 9)):
    o = (C.c_int32 * 3)(*orig)
    d = (C.c_uint32 * 3)(*dims)
    rc = lib_abi.tsp_b200_try_build_cell_frame((C.c_int64 * 3)(*lo), (C.c_int64 * 3)(*hi), o, d)
    return rc, tuple(o), tuple(d)


@pytest.fixture(scope="module")
def lib_abi():
    if not os.path.exists(abi.LIB_PATH):
        from turbospharticles_b200 import build
        build.build()
    return abi.load_library()


def test_cell_frame_inclusive_signed_bounds(lib_abi):
    rc, o, d = _frame(lib_abi, (-3, 5, -7), (1, 6, -7))
    assert rc == 0 and o == (-3, 5, -7) and d == (5, 2, 1)


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_cell_frame_maximum_axis_extent(lib_abi, axis):
    hi = [0, 0, 0]
    hi[axis] = 2_097_151
    rc, o, d = _frame(lib_abi, (0, 0, 0), hi)
    want = [1, 1, 1]
    want[axis] = 2_097_152
    assert rc == 0 and d == tuple(want)


@pytest.mark.parametrize("b", [
    (1, 0, 0, 0, 0, 0), (0, 1, 0, 0, 0, 0), (0, 0, 1, 0, 0, 0),
    (-2_147_483_649, 0, 0, -2_147_483_649, 0, 0), (0, -2_147_483_649, 0, 0, -2_147_483_649, 0),
    (0, 0, -2_147_483_649, 0, 0, -2_147_483_649),
    (2_147_483_648, 0, 0, 2_147_483_648, 0, 0), (0, 2_147_483_648, 0, 0, 2_147_483_648, 0),
    (0, 0, 2_147_483_648, 0, 0, 2_147_483_648),
    (0, 0, 0, 2_097_152, 0, 0), (0, 0, 0, 0, 2_097_152, 0), (0, 0, 0, 0, 0, 2_097_152)])
def test_cell_frame_invalid_bounds_preserve_frame(lib_abi, b):
    rc, o, d = _frame(lib_abi, b[:3], b[3:])
    assert rc == -4  # TSP_ERR_FRAME
    assert o == (4, 5, 6) and d == (7, 8, 9)


def test_batch_scene_bytes_is_host_arithmetic(lib_abi):
    f = lib_abi.tsp_b200_batch_scene_bytes
    a = f(4096, 5000, 100_000)
    assert a > 0
    assert f(8192, 5000, 100_000) > a          # more fluid costs more
    assert f(4096, 10000, 100_000) > a         # more boundary costs more
    assert f(4096, 5000, 200_000) > a          # a larger frame costs more
    assert f(4095, 5000, 100_000) == a         # fluid is charged in whole 32-particle chunks
