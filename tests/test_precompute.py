"""Host set-up of the library (lumped mass, rest volume, Dm^-1, V0) is bit-exact with the
oracle's restatement of TetMesh::initialize and VBDsolver::precomputeTetData."""
import numpy as np
import pytest

from oracle import pyoracle as po
from vbd_tetmesh_b200 import mesh_mass, meshgen, precompute_tets


@pytest.mark.parametrize("mesh", ["beam", "block", "cube16"])
def test_setup_bit_exact(mesh):
    m = {"beam": meshgen.beam, "block": lambda: meshgen.jittered_block(7, 3, 4, seed=5),
         "cube16": lambda: meshgen.cube(16)}[mesh]()
    mass, vol = mesh_mass(m.rest, m.tets, m.density)
    dm, v0 = precompute_tets(m.rest, m.tets)
    mo, trv, dmo, v0o = po.mesh_setup(m.rest, m.tets, m.density, precision=32)
    np.testing.assert_array_equal(mass.astype(np.float64), mo)
    np.testing.assert_array_equal(vol.astype(np.float64), trv)
    np.testing.assert_array_equal(dm.astype(np.float64), dmo)
    np.testing.assert_array_equal(v0.astype(np.float64), v0o)


def test_mass_sums_to_density_times_volume():
    m = meshgen.jittered_block(5, 5, 5, seed=2, jitter=0.0)
    mass, vol = mesh_mass(m.rest, m.tets, m.density)
    assert abs(mass.sum() - m.density * vol.sum()) < 1e-4 * mass.sum()
    assert abs(vol.sum() - 5 ** 3 * 0.05 ** 3) < 1e-6


def test_dminv_inverts_rest_edges():
    m = meshgen.jittered_block(3, 3, 3, seed=4)
    dm, v0 = precompute_tets(m.rest, m.tets)
    r = m.rest.astype(np.float64)
    D = np.stack([r[m.tets[:, k]] - r[m.tets[:, 0]] for k in (1, 2, 3)], axis=2)
    eye = np.einsum("tij,tjk->tik", D, dm.astype(np.float64))
    assert np.abs(eye - np.eye(3)).max() < 1e-5
    np.testing.assert_allclose(v0, np.abs(np.linalg.det(D)) / 6.0, rtol=1e-5)


def test_cube_min_volume_positive():
    m = meshgen.cube(64)
    _, v0 = precompute_tets(m.rest, m.tets)
    assert v0.min() > 0.0
