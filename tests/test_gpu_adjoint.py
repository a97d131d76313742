"""Hand-written adjoint (implicit differentiation of each converged step) through the C ABI:
against the FP64 oracle adjoint, against central finite differences of the FP64 forward,
checkpoint-interval invariance, state preservation, and the torch autograd shim."""
import numpy as np
import pytest

from oracle import pyoracle as po
from vbd_tetmesh_b200 import build_solver, meshgen

pytestmark = pytest.mark.gpu

GRAD_RTOL = 1e-3


def rel(a, b):
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def setup_case(seed=1):
    m = meshgen.jittered_block(3, 2, 2, seed=seed, per_tet_sigma=0.2, E=2e4)
    W = np.random.default_rng(seed).normal(size=(m.num_verts, 3))
    return m, W


def gpu_grads(m, W, steps, dt, iters, accel, rho, checkpoint, adj_iters):
    s = build_solver(m)
    s.record(checkpoint)
    for _ in range(steps):
        s.step(dt, iters, (0.0, -9.8, 0.0), accel, rho)
    x_before = s.get_positions()
    g = s.backward(W, None, adj_iters)
    assert np.array_equal(s.get_positions(), x_before), "backward changed the solver state"
    s.close()
    return g


def test_adjoint_matches_fp64_oracle(gpu_device):
    m, W = setup_case()
    steps, dt, iters = 3, 1 / 60, 300
    gx, gv, gm, gl = gpu_grads(m, W, steps, dt, iters, False, 0.0, 2, 300)
    o = po.adjoint_f64(m, steps, dt, iters, lambda x: W, use_acceleration=False)
    errs = dict(mu=rel(gm, o["gmu"]), lam=rel(gl, o["glam"]), x0=rel(gx, o["gx0"]), v0=rel(gv, o["gv0"]))
    print("GPU adjoint vs FP64 adjoint (relative L2):", errs, "oracle CG residual", o["residual"])
    assert all(e < GRAD_RTOL for e in errs.values()), errs


def test_adjoint_matches_finite_differences(gpu_device):
    m, W = setup_case(seed=2)
    steps, dt, iters = 3, 1 / 60, 300
    gx, gv, gm, gl = gpu_grads(m, W, steps, dt, iters, False, 0.0, 3, 300)
    L = lambda x: float(np.sum(W * x))  # noqa: E731

    def fd(param, idx, comp=0):
        def run(sign):
            mu, lam = m.mu.astype(float).copy(), m.lam.astype(float).copy()
            x0, v0 = m.x.astype(float).copy(), m.v.astype(float).copy()
            if param == "mu":
                d = 1e-4 * mu[idx]
                mu[idx] += sign * d
            elif param == "lam":
                d = 1e-4 * lam[idx]
                lam[idx] += sign * d
            elif param == "x0":
                d = 1e-6
                x0[idx, comp] += sign * d
            else:
                d = 1e-4
                v0[idx, comp] += sign * d
            x = po.adjoint_f64(m, steps, dt, iters, None, use_acceleration=False, mu=mu, lam=lam, x0=x0, v0=v0)["x"]
            return L(x), d

        (lp, d), (lm, _) = run(1.0), run(-1.0)
        return (lp - lm) / (2 * d)

    rng = np.random.default_rng(5)
    checks = []
    for e in rng.choice(m.num_tets, 4, replace=False):
        checks += [("mu", int(e), 0, gm[e]), ("lam", int(e), 0, gl[e])]
    free = np.flatnonzero(m.fixed == 0)
    for vtx in rng.choice(free, 3, replace=False):
        checks += [("x0", int(vtx), 1, gx[vtx, 1]), ("v0", int(vtx), 2, gv[vtx, 2])]
    checks += [("x0", int(np.flatnonzero(m.fixed == 1)[0]), 0, gx[np.flatnonzero(m.fixed == 1)[0], 0])]
    scale = {k: max(abs(c[3]) for c in checks if c[0] == k) for k in ("mu", "lam", "x0", "v0")}
    for param, idx, comp, g in checks:
        ref = fd(param, idx, comp)
        err = abs(g - ref) / max(abs(ref), 1e-3 * scale[param])
        print(f"{param}[{idx}]: adjoint {g:.6e} fd {ref:.6e} rel {err:.2e}")
        assert err < GRAD_RTOL


def test_checkpoint_interval_does_not_change_gradients(gpu_device):
    m, W = setup_case(seed=3)
    ref = gpu_grads(m, W, 6, 1 / 60, 20, True, 0.9, 1, 40)
    for k in (2, 4, 6):
        g = gpu_grads(m, W, 6, 1 / 60, 20, True, 0.9, k, 40)
        for a, b in zip(g, ref):
            np.testing.assert_array_equal(a, b)


def test_autograd_shim(gpu_device):
    import torch

    from autograd_shim import VBDRollout

    m, W = setup_case(seed=4)
    s = build_solver(m)
    mu = torch.tensor(m.mu, dtype=torch.float64, requires_grad=True)
    lam = torch.tensor(m.lam, dtype=torch.float64, requires_grad=True)
    x0 = torch.tensor(m.x, dtype=torch.float64, requires_grad=True)
    v0 = torch.tensor(m.v, dtype=torch.float64, requires_grad=True)
    xT = VBDRollout.apply(mu, lam, x0, v0, s, 3, 1 / 60, 300, (0.0, -9.8, 0.0), False, 0.0, 2, 300)
    loss = (torch.from_numpy(W) * xT).sum()
    loss.backward()
    o = po.adjoint_f64(m, 3, 1 / 60, 300, lambda x: W, use_acceleration=False)
    assert rel(mu.grad.numpy(), o["gmu"]) < GRAD_RTOL
    assert rel(lam.grad.numpy(), o["glam"]) < GRAD_RTOL
    assert rel(x0.grad.numpy(), o["gx0"]) < GRAD_RTOL
    assert rel(v0.grad.numpy(), o["gv0"]) < GRAD_RTOL
