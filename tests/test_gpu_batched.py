"""Batched many-mesh mode: one solver over concatenated meshes (per-mesh offsets, colour c of every
mesh in one launch) gives each mesh bit-identically what its own solver gives, and stays within the
parity bar of the FP32 oracle and the stated error of the FP64 oracle for every mesh."""
import numpy as np
import pytest

from helpers import rel_err
from oracle import pyoracle as po
from vbd_tetmesh_b200 import VBDError, build_batch_solver, build_solver, meshgen

pytestmark = pytest.mark.gpu


def small_batch():
    return meshgen.batched_blocks(num_meshes=6, lo=2, hi=6, seed=7)


@pytest.mark.parametrize("layout", [1, 2, 3, 4])
def test_batch_bit_identical_to_per_mesh_solvers(gpu_device, layout):
    meshes = small_batch()
    b = meshgen.concat(meshes)
    s = build_batch_solver(b)
    from vbd_tetmesh_b200 import _capi

    s.set_option(_capi.OPT_LAYOUT, layout)
    for _ in range(5):
        s.step(1 / 60, 20, (0.0, -9.8, 0.0), True, 0.9)
    xb = b.split(s.get_positions())
    vb = b.split(s.get_velocities())
    lanes = s.get_option(_capi.OPT_LANES)  # the per-mesh solvers run the batch's launch shape
    for m, x, v in zip(meshes, xb, vb):
        p = build_solver(m, layout=layout, lanes=lanes)
        for _ in range(5):
            p.step(1 / 60, 20, (0.0, -9.8, 0.0), True, 0.9)
        np.testing.assert_array_equal(x, p.get_positions())
        np.testing.assert_array_equal(v, p.get_velocities())
        p.close()


def test_batch_matches_oracle_per_mesh(gpu_device):
    meshes = small_batch()
    b = meshgen.concat(meshes)
    s = build_batch_solver(b)
    for _ in range(10):
        s.step(1 / 60, 20, (0.0, -9.8, 0.0), True, 0.9)
    for m, x in zip(meshes, b.split(s.get_positions())):
        o32 = po.simulate(m, 10, 1 / 60, 20, (0.0, -9.8, 0.0), True, 0.9, precision=32)
        o64 = po.simulate(m, 10, 1 / 60, 20, (0.0, -9.8, 0.0), True, 0.9, precision=64, mode=po.CLOSED)
        e32, e64 = rel_err(x, o32["x"], m), rel_err(x, o64["x"], m)
        print(f"mesh {m.dims}: vs oracle32 {e32:.2e} vs oracle64 {e64:.2e}")
        assert e32 < 1e-5 and e64 < 1e-5


def test_batch_rejects_ids_outside_their_mesh(gpu_device):
    meshes = small_batch()[:2]
    b = meshgen.concat(meshes)
    b.tets_local = b.tets_local.copy()
    b.tets_local[b.tet_offsets[1], 0] = meshes[1].num_verts + 3
    with pytest.raises(VBDError) as e:
        build_batch_solver(b)
    assert "mesh 1" in e.value.message
