"""Batched material identification (many meshes, one solver, forward + adjoint per outer step)."""
import numpy as np
import pytest

from oracle import pyoracle as po
from vbd_tetmesh_b200 import material_id as mid

pytestmark = pytest.mark.gpu

GRAD_RTOL = 1e-3  # the adjoint's bar against finite differences


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
    prob.solver.close()


def _oracle_loss(m, logE, nu, target, st):
    """The FP64 oracle's forward of one beam from rest with (E, nu) on every tet, and its loss."""
    E = np.exp(logE)
    mu, lam, _, _ = mid.lame_and_derivatives(E, nu)
    T = m.num_tets
    x = po.adjoint_f64(m, st.steps, st.dt, st.iterations, None, gravity=st.gravity, use_acceleration=True,
                       rho=st.rho, x0=m.rest, v0=np.zeros_like(m.rest), mu=np.full(T, mu), lam=np.full(T, lam))["x"]
    return float(np.sum((x - target) ** 2))


def test_per_mesh_gradients_match_fp64_finite_differences(gpu_device):
    """With every step's forward converged (200 iterations), the batched adjoint's per-mesh
    d(loss)/d(log E) and d(loss)/d(nu) match central finite differences of the FP64 oracle's forward
    of each mesh on its own (step 1e-4 in log E, 1e-4 nu in nu) within 1e-3, at a point away from
    the hidden parameters."""
    meshes, hidden = small_problem()
    st = mid.Settings(steps=6, iterations=200, adjoint_iterations=150)
    prob = mid.Problem.create(meshes, st)
    targets = prob.forward(np.log(hidden[:, 0]), hidden[:, 1])
    lE = np.log(hidden[:, 0]) + 0.4
    nu = hidden[:, 1] - 0.06
    _, gE, gN = prob.loss_and_grad(lE, nu, targets)
    prob.solver.close()
    errs = []
    for k, m in enumerate(meshes):
        tk = targets[prob.batch.vert_offsets[k]:prob.batch.vert_offsets[k + 1]]
        h = 1e-4
        fE = (_oracle_loss(m, lE[k] + h, nu[k], tk, st) - _oracle_loss(m, lE[k] - h, nu[k], tk, st)) / (2 * h)
        hn = 1e-4 * nu[k]
        fN = (_oracle_loss(m, lE[k], nu[k] + hn, tk, st) - _oracle_loss(m, lE[k], nu[k] - hn, tk, st)) / (2 * hn)
        eE, eN = abs(gE[k] - fE) / abs(fE), abs(gN[k] - fN) / abs(fN)
        print(f"mesh {k} dims {m.dims}: dL/dlogE adjoint {gE[k]:.6e} fd64 {fE:.6e} rel {eE:.2e}; "
              f"dL/dnu adjoint {gN[k]:.6e} fd64 {fN:.6e} rel {eN:.2e}")
        errs += [eE, eN]
    assert max(errs) < GRAD_RTOL, errs


def test_identification_recovers_hidden_materials(gpu_device):
    meshes, hidden = small_problem()
    prob = mid.Problem.create(meshes, mid.Settings(steps=10))
    targets = prob.forward(np.log(hidden[:, 0]), hidden[:, 1])
    lE0 = np.full(len(meshes), np.log(1e5))
    nu0 = np.full(len(meshes), 0.3)
    logE, nu, hist, final = mid.identify(prob, targets, lE0, nu0, outer=30)
    prob.solver.close()
    relE = np.abs(np.exp(logE) / hidden[:, 0] - 1.0)
    dnu = np.abs(nu - hidden[:, 1])
    print(f"loss {hist[0]:.4e} -> {hist[-1]:.4e}; E rel err {relE}, nu abs err {dnu}, final losses {final}")
    assert hist[-1] < 1e-3 * hist[0]
    assert np.all(np.diff(hist) <= 0.0)  # every accepted step lowers the loss
    assert relE.max() < 0.05
