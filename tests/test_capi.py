"""The C-ABI library loads, exports every entry point that include/vbd_b200.h declares, and its
host-side calls follow the error convention (no GPU needed)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from vbd_tetmesh_b200 import _capi
from vbd_tetmesh_b200._capi import VBDError, lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "vbd_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(vbd_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_functions():
    names = declared_functions()
    assert "vbd_solver_step" in names and "vbd_color_vertices" in names
    assert len(names) >= 25


def test_library_exports_every_declared_symbol():
    L = lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, f"symbols declared in vbd_b200.h but not exported: {missing}"


def test_python_binding_covers_header():
    assert set(declared_functions()) <= set(_capi.SIGNATURES)


def test_version_and_error_string():
    assert lib().vbd_version() >= 100
    assert isinstance(lib().vbd_last_error(), bytes)


def test_colouring_rejects_out_of_range_ids():
    tets = np.array([[0, 1, 2, 7]], np.int32)
    out = np.empty(4, np.int32)
    nc = C.c_int32()
    rc = lib().vbd_color_vertices(4, 1, tets.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p),
                                  C.byref(nc), 0, None, None)
    assert rc == 1
    assert b"outside" in lib().vbd_last_error()


def test_colouring_rejects_repeated_ids():
    tets = np.array([[0, 1, 1, 2]], np.int32)
    from vbd_tetmesh_b200 import color_vertices

    with pytest.raises(VBDError) as e:
        color_vertices(3, tets)
    assert e.value.code == 1 and "repeats" in e.value.message


def test_colour_group_capacity_is_checked():
    from vbd_tetmesh_b200 import meshgen

    m = meshgen.beam(4, 2, 2)
    out = np.empty(m.num_verts, np.int32)
    offs = np.empty(3, np.int32)
    verts = np.empty(m.num_verts, np.int32)
    nc = C.c_int32()
    rc = lib().vbd_color_vertices(m.num_verts, m.num_tets, m.tets.ctypes.data_as(C.c_void_p),
                                  out.ctypes.data_as(C.c_void_p), C.byref(nc), 2, offs.ctypes.data_as(C.c_void_p),
                                  verts.ctypes.data_as(C.c_void_p))
    assert rc == 1 and b"capacity" in lib().vbd_last_error()


def test_null_handle_is_rejected():
    rc = lib().vbd_solver_step(None, 0.01, 1, 1, None, 0, 0.0)
    assert rc == 1
    assert lib().vbd_solver_destroy(None) == 0


def test_create_without_b200_reports_no_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present; covered by the GPU tests")
    h = C.c_void_p()
    rc = lib().vbd_solver_create(C.byref(h), 0, None)
    assert rc == 5, _capi.STATUS_NAMES.get(rc)
    assert not h.value
