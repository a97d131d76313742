"""A TetGen-loaded mesh (the reference driver's input path) simulated on the GPU: the rest shape from
block1.node, the pre-compressed current shape from block1_cur.node, the bottom 5% in y pinned, as
main.cpp sets up its meshes; checked against the oracle under both semantics."""
import os

import numpy as np
import pytest

from helpers import gpu_simulate, rel_err
from oracle import pyoracle as po
from vbd_tetmesh_b200 import _capi, build_solver, surface, tetgen

pytestmark = pytest.mark.gpu

GOLD_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tetgen")


def load():
    return tetgen.load_tetgen(os.path.join(GOLD_DIR, "block1.node"), os.path.join(GOLD_DIR, "block1.ele"),
                              os.path.join(GOLD_DIR, "block1_cur.node"), density=1000.0, E=1e5, nu=0.3)


def test_tetgen_mesh_vbdsolver_semantics(gpu_device):
    m = load()
    assert m.fixed.sum() > 0
    g = gpu_simulate(m, 5, 1 / 60, 20, (0.0, 0.0, 0.0), True, 0.75)
    o = po.simulate(m, 5, 1 / 60, 20, (0.0, 0.0, 0.0), True, 0.75, precision=32)
    err = rel_err(g["x"], o["x"], m)
    print(f"TetGen block, 5 steps from the compressed shape: |gpu - oracle32|/diag = {err:.2e}")
    assert err < 1e-5
    # the compressed block relaxes toward its rest shape
    assert np.abs(g["x"] - m.rest).max() < np.abs(m.x - m.rest).max()
    # OBJ export of the device readback (TetMesh::exportToObj's text)
    text = surface.obj_text(g["x"], m.tets)
    assert text.count("\nv ") == m.num_verts
    assert text.count("\nf ") == len(surface.extract_surface_faces(m.tets)) > 0


def test_tetgen_mesh_wrapper_semantics(gpu_device):
    m = load()
    s = build_solver(m)
    s.set_option(_capi.OPT_SEMANTICS, 1)
    for _ in range(5):
        s.step(1 / 60, 20, (0.0, 0.0, 0.0), True, 0.75)
    x = s.get_positions()
    s.close()
    o = po.simulate(m, 5, 1 / 60, 20, (0.0, 0.0, 0.0), True, 0.75, precision=32, mode=po.WRAPPER)
    assert rel_err(x, o["x"], m) < 1e-5
