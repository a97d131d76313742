"""Batched material identification (many meshes, one solver, forward + adjoint per outer step)."""
import numpy as np
import pytest

from vbd_tetmesh_b200 import material_id as mid

pytestmark = pytest.mark.gpu


def small_problem(n=6):
    meshes, hidden = mid.beams(n, seed=5)
    meshes = [m for m in meshes if m.num_verts < 1500][:4]
    hidden = np.array([(m.meta["E"], m.meta["nu"]) for m in meshes])
    return meshes, hidden


def test_batched_gradients_equal_per_mesh_gradients(gpu_device):
    meshes, hidden = small_problem()
    st = mid.Settings(steps=5, iterations=40, adjoint_iterations=30)
    prob = mid.Problem.create(meshes, st)
    targets = prob.forward(np.log(hidden[:, 0]), hidden[:, 1])
    lE = np.log(hidden[:, 0]) + 0.3
    nu = hidden[:, 1] - 0.05
    L, gE, gN = prob.loss_and_grad(lE, nu, targets)
    for k, m in enumerate(meshes):
        one = mid.Problem.create([m], st)
        tk = targets[prob.batch.vert_offsets[k]:prob.batch.vert_offsets[k + 1]]
        Lk, gEk, gNk = one.loss_and_grad(lE[k:k + 1], nu[k:k + 1], tk)
        np.testing.assert_allclose(L[k], Lk[0], rtol=1e-12)
        np.testing.assert_allclose(gE[k], gEk[0], rtol=1e-9)
        np.testing.assert_allclose(gN[k], gNk[0], rtol=1e-9)
        one.solver.close()


def test_gradients_match_finite_differences_and_descent_reduces_loss(gpu_device):
    meshes, hidden = small_problem()
    prob = mid.Problem.create(meshes, mid.Settings(steps=10))
    targets = prob.forward(np.log(hidden[:, 0]), hidden[:, 1])
    lE0 = np.full(len(meshes), np.log(1e5))
    nu0 = np.full(len(meshes), 0.3)
    _, gE, gN = prob.loss_and_grad(lE0, nu0, targets)
    fE = prob.fd_grad(lE0, nu0, targets, "logE", 1e-3)
    assert np.median(np.abs(gE - fE) / np.abs(fE)) < 1e-2
    _, _, hist = mid.identify(prob, targets, lE0, nu0, outer=10)
    assert hist[-1] < 0.5 * hist[0]
