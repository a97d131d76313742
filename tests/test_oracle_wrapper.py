"""The oracle's restatement of the reference GPU wrapper's semantics (mode WRAPPER: corotated element
of VBD_DeviceMath.cuh:127-198, vbd_solve_color_kernel's update of VBD_GPU_Wrapper.cu:114-235,
solveVBD's loop of :332-362), pinned on the CPU:
  * the corotated block against an independent float64 evaluation (polar factor from an SVD);
  * whole runs against tests/golden/wrapper_ref.npz, outputs of the reference's own GPU kernels
    (VBD_GPU_Solver built from its sources, tests/golden/make_wrapper_golden.py)."""
import os

import numpy as np
import pytest

from helpers import rel_err
from oracle import pyoracle as po
from vbd_tetmesh_b200 import meshgen

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "wrapper_ref.npz")
POS_TOL = 1e-5  # of the bounding-box diagonal


def corot_numpy(F, dminv, mu, lam, vol, n):
    U, _, Vt = np.linalg.svd(F)
    R = U @ Vt
    tr = np.sum(R * F) - 3.0
    P = 2.0 * mu * (F - R) + lam * tr * R
    q = -dminv.sum(axis=0) if n == 0 else dminv[n - 1]
    g = vol * P @ q
    rq = R @ q
    H = vol * (2.0 * mu * (q @ q) * np.eye(3) + lam * np.outer(rq, rq))
    return H, g


@pytest.mark.parametrize("seed", range(6))
def test_corotated_block_matches_svd_polar_factor(seed):
    rng = np.random.default_rng(seed)
    # a rotation times a moderate stretch (singular values in [0.8, 1.25]): 5 Higham steps converge
    Q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    if np.linalg.det(Q) < 0:
        Q[:, 0] *= -1
    S = np.diag(rng.uniform(0.8, 1.25, 3))
    V, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    F = Q @ V @ S @ V.T
    dminv = rng.normal(size=(3, 3)) * 20.0
    mu, lam, vol = 3.8e4, 5.7e4, 1e-4
    for n in range(4):
        H, g = po.tet_block(F, dminv, mu, lam, vol, n, mode=po.WRAPPER, precision=64)
        Hr, gr = corot_numpy(F, dminv, mu, lam, vol, n)
        assert np.abs(H - Hr).max() <= 1e-9 * np.abs(Hr).max()
        assert np.abs(g - gr).max() <= 1e-9 * max(np.abs(gr).max(), 1e-30)


def test_corotated_block_at_rest_has_no_force():
    dminv = np.diag([20.0, 20.0, 20.0])
    for n in range(4):
        H, g = po.tet_block(np.eye(3), dminv, 1e4, 2e4, 1e-3, n, mode=po.WRAPPER, precision=64)
        assert np.abs(g).max() == 0.0
        assert np.allclose(H, H.T)


def _frames_oracle(m, dt, iters, rho, frames, precision):
    return po.simulate(m, frames, dt, iters, (0.0, -9.8, 0.0), True, rho, precision=precision, mode=po.WRAPPER,
                       v0=np.zeros_like(m.x))


@pytest.mark.parametrize("case,frames", [("beam", 1), ("beam", 5), ("cube6", 1), ("cube6", 3)])
def test_wrapper_oracle_matches_reference_gpu_outputs(case, frames):
    gold = np.load(GOLDEN)
    if case == "beam":
        m, dt, iters, rho = meshgen.beam(), 1.0 / 60.0, 20, 0.95
    else:
        m, dt, iters, rho = meshgen.cube(6, E=1e6, nu=0.4, seed=5), 1.0 / 120.0, 50, 0.9
    ref = gold[f"{case}/x_f{frames}"]
    o32 = _frames_oracle(m, dt, iters, rho, frames, 32)
    o64 = _frames_oracle(m, dt, iters, rho, frames, 64)
    e32, e64 = rel_err(o32["x"], ref, m), rel_err(o64["x"], ref, m)
    print(f"{case} {frames} frames: oracle32 vs reference GPU {e32:.2e}, oracle64 vs reference GPU {e64:.2e}")
    assert e32 < POS_TOL
    vscale = max(np.abs(gold[f"{case}/v_f{frames}"]).max(), 1e-6)
    assert np.abs(o32["v"] - gold[f"{case}/v_f{frames}"]).max() < 1e-3 * vscale


@pytest.mark.parametrize("accel", [0, 1])
def test_wrapper_oracle_solve_matches_reference_gpu(accel):
    gold = np.load(GOLDEN)
    m = meshgen.jittered_block(6, 4, 5, seed=3)
    x = po.solve(m, m.x, gold["solve/y"], 3600.0, 30, bool(accel), 0.9, init_from_inertia=True, mode=po.WRAPPER)
    err = rel_err(x, gold[f"solve/x_accel{accel}"], m)
    print(f"solveVBD accel={accel}: oracle32 vs reference GPU {err:.2e}")
    assert err < POS_TOL
