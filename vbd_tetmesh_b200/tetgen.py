"""TetGen meshes (.node / .ele) as the reference's driver loads them (main.cpp:14-168).

Parsing and pinning run in libvbd_b200.so (``vbd_tetgen_read_node``, ``vbd_tetgen_read_ele``,
``vbd_pin_low_fraction``), the same code the C++ header ``include/vbd/TetGenIO.h`` calls, so both
read a file identically.  :func:`load_tetgen` returns a :class:`meshgen.Mesh` ready for
``build_solver``; :func:`write_tetgen` writes one out (for tests and round trips).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import meshgen
from ._capi import VBDError, call
from .solver import _ptr

AXES = {"x": 0, "y": 1, "z": 2}


def read_node(path):
    """(positions (N, 3) float32, index of the first node)."""
    n = C.c_int32(0)
    first = C.c_int32(0)
    call("vbd_tetgen_read_node", os.fsencode(path), C.byref(n), None, None, 0)
    pos = np.empty((n.value, 3), np.float32)
    call("vbd_tetgen_read_node", os.fsencode(path), C.byref(n), C.byref(first), _ptr(pos), n.value)
    return pos, first.value


def read_ele(path, index_base, num_nodes=-1):
    """Element vertex ids (T, 4) int32, shifted down by index_base (0 or 1)."""
    t = C.c_int32(0)
    call("vbd_tetgen_read_ele", os.fsencode(path), int(index_base), int(num_nodes), C.byref(t), None, 0)
    tets = np.empty((t.value, 4), np.int32)
    call("vbd_tetgen_read_ele", os.fsencode(path), int(index_base), int(num_nodes), C.byref(t), _ptr(tets), t.value)
    return tets


def pin_low_fraction(positions, axis, fraction=0.05, fixed=None):
    """Marks vertices whose coordinate on ``axis`` is within ``fraction`` of the extent above the
    minimum (main.cpp:127-163); returns the uint8 flags (``fixed`` is updated in place if given)."""
    pos = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
    out = np.zeros(pos.shape[0], np.uint8) if fixed is None else fixed
    ax = AXES[axis] if isinstance(axis, str) else int(axis)
    call("vbd_pin_low_fraction", pos.shape[0], _ptr(pos), ax, float(fraction), _ptr(out))
    return out


def lame_f32(E, nu):
    """(mu, lambda) computed in float32 as main.cpp:173-174 does."""
    E, nu = np.float32(E), np.float32(nu)
    one, two = np.float32(1.0), np.float32(2.0)
    mu = E / (two * (one + nu))
    lam = E * nu / ((one + nu) * (one - two * nu))
    return float(mu), float(lam)


def load_tetgen(rest_node, ele, current_node=None, density=7800.0e-12, E=200.0e3, nu=0.3, mu=None, lam=None,
                pin_axes=("y",), pin_fraction=0.05) -> meshgen.Mesh:
    """The reference driver's loadTetgenModel (main.cpp:48-168).

    Rest positions come from ``rest_node``; the current (initial) positions from ``current_node``,
    or the rest positions when it is None or missing (main.cpp:66-71).  Ids are 0-based when the
    rest file's first node index is 0, else 1-based.  Vertices within ``pin_fraction`` of the
    extent above the minimum of each axis in ``pin_axes`` (measured on the current positions) are
    pinned; main.cpp pins along y only.  The defaults are main.cpp's material (E = 200e3,
    nu = 0.3, density 7800e-12, millimetre units); ``mu`` / ``lam`` override E / nu."""
    rest, first = read_node(rest_node)
    if rest.shape[0] == 0:
        raise VBDError("vbd_tetgen_read_node", 1, f"'{rest_node}': no nodes")
    base = 0 if first == 0 else 1
    if current_node is not None and os.path.exists(current_node):
        cur, _ = read_node(current_node)
        if cur.shape[0] != rest.shape[0]:
            raise VBDError("vbd_tetgen_read_node", 1,
                           f"rest nodes ({rest.shape[0]}) and current nodes ({cur.shape[0]}) count mismatch")
    else:
        cur = rest.copy()
    tets = read_ele(ele, base, rest.shape[0])
    fixed = np.zeros(rest.shape[0], np.uint8)
    for ax in pin_axes:
        pin_low_fraction(cur, ax, pin_fraction, fixed)
    if mu is None or lam is None:
        mu, lam = lame_f32(E, nu)
    t = tets.shape[0]
    return meshgen.Mesh(rest=rest, x=cur.copy(), v=np.zeros_like(rest), tets=tets, fixed=fixed,
                        mu=np.full(t, mu, np.float32), lam=np.full(t, lam, np.float32), density=float(density),
                        meta=dict(kind="tetgen", rest_node=str(rest_node), ele=str(ele), index_base=base))


def write_tetgen(path_prefix, positions, tets, index_base=1, node_suffix=".node", comment=True):
    """Writes ``<prefix>.node`` (positions) and ``<prefix>.ele`` (tets) in TetGen's format with ids
    starting at ``index_base``; floats are written with enough digits to read back exactly."""
    pos = np.asarray(positions, np.float32).reshape(-1, 3)
    tets = np.asarray(tets, np.int64).reshape(-1, 4)
    node_path, ele_path = f"{path_prefix}{node_suffix}", f"{path_prefix}.ele"
    with open(node_path, "w") as f:
        f.write(f"{pos.shape[0]}  3  0  0\n")
        for i, p in enumerate(pos):
            f.write(f"   {i + index_base}    {float(p[0])!r}  {float(p[1])!r}  {float(p[2])!r}\n")
        if comment:
            f.write("# written by vbd_tetmesh_b200.tetgen\n")
    with open(ele_path, "w") as f:
        f.write(f"{tets.shape[0]}  4  0\n")
        for t, q in enumerate(tets):
            f.write(f"   {t + index_base}    {q[0] + index_base}  {q[1] + index_base}  {q[2] + index_base}  "
                    f"{q[3] + index_base}\n")
        if comment:
            f.write("# written by vbd_tetmesh_b200.tetgen\n")
    return node_path, ele_path
