"""Batched material identification: recover per-mesh (log E, nu) from final positions.

Every mesh of the batch advances in one solver (colour c of all meshes in one launch); one
recorded forward and one backward pass (vbd_solver_record / vbd_solver_backward) give the
per-tet gradients dL/dmu, dL/dlambda of the loss L = sum_m sum_i |x_i - x*_i|^2, which chain to
each mesh's (log E, nu) through mu = E / (2 (1 + nu)), lambda = E nu / ((1 + nu)(1 - 2 nu)).
Each mesh's (log E, nu) moves by its own trust-region step (identify: quasi-Newton on the
adjoint's gradients, or Levenberg-Marquardt on a finite-difference Jacobian); one trial of all
meshes costs one batched forward + adjoint.  Finite-difference checks need only two
batched forwards per parameter, since the meshes are independent.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import meshgen
from .solver import build_batch_solver


def beams(num=64, seed=77, cell=0.05):
    """The material-identification configuration: `num` beams with Lx ~ U{8..40}, Ly = Lz ~ U{3..8}
    (6 tets per cell, x = 0 face pinned) and hidden (E, nu): E log-uniform in [1e4, 1e6] Pa, nu
    uniform in [0.2, 0.45]."""
    rng = np.random.default_rng(seed)
    meshes, hidden = [], []
    for _ in range(num):
        lx = int(rng.integers(8, 41))
        ly = int(rng.integers(3, 9))
        E = float(10.0 ** rng.uniform(4.0, 6.0))
        nu = float(rng.uniform(0.2, 0.45))
        meshes.append(meshgen.beam(lx, ly, ly, cell=cell, E=E, nu=nu))
        hidden.append((E, nu))
    return meshes, np.array(hidden)


def lame_and_derivatives(E, nu):
    """(mu, lambda, dmu/dnu, dlambda/dnu) of E, nu (arrays)."""
    mu = E / (2.0 * (1.0 + nu))
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    dmu = -E / (2.0 * (1.0 + nu) ** 2)
    dlam = E * (1.0 + 2.0 * nu * nu) / ((1.0 + nu) ** 2 * (1.0 - 2.0 * nu) ** 2)
    return mu, lam, dmu, dlam


@dataclass
class Settings:
    steps: int = 20
    dt: float = 1.0 / 60.0
    iterations: int = 100
    rho: float = 0.95
    gravity: tuple = (0.0, -9.8, 0.0)
    checkpoint: int = 10
    adjoint_iterations: int = 50
    adjoint_rho: float = 0.95


@dataclass
class Problem:
    """A batch of meshes, its solver and the per-tet mesh index."""

    batch: meshgen.Batch
    solver: object
    tet_mesh: np.ndarray
    settings: Settings = field(default_factory=Settings)
    last_x: np.ndarray | None = None

    @classmethod
    def create(cls, meshes, settings=None, device=0, stream=None):
        b = meshgen.concat(meshes)
        s = build_batch_solver(b, device=device, stream=stream)
        tet_mesh = np.repeat(np.arange(len(meshes)), np.diff(b.tet_offsets))
        return cls(b, s, tet_mesh, settings or Settings())

    def _materials(self, logE, nu):
        E = np.exp(np.asarray(logE, np.float64))[self.tet_mesh]
        n = np.asarray(nu, np.float64)[self.tet_mesh]
        mu, lam, dmu, dlam = lame_and_derivatives(E, n)
        return mu, lam, dmu, dlam

    def forward(self, logE, nu, record=False):
        """Final positions after `steps` steps from rest with per-mesh (log E, nu); also kept in
        self.last_x (loss_and_grad runs one forward)."""
        st = self.settings
        mu, lam, _, _ = self._materials(logE, nu)
        s = self.solver
        s.set_materials(mu.astype(np.float32), lam.astype(np.float32))
        s.set_positions(self.batch.rest)
        s.set_velocities(np.zeros_like(self.batch.rest))
        s.record(st.checkpoint if record else 0)
        for _ in range(st.steps):
            s.step(st.dt, st.iterations, st.gravity, True, st.rho)
        self.last_x = s.get_positions().astype(np.float64)
        return self.last_x

    def losses(self, x, targets):
        """Per-mesh loss sum_i |x_i - x*_i|^2."""
        d2 = np.sum((x - targets) ** 2, axis=1)
        return np.add.reduceat(d2, self.batch.vert_offsets[:-1])

    def loss_and_grad(self, logE, nu, targets):
        """Per-mesh losses and gradients w.r.t. (log E, nu), from one forward and one backward."""
        st = self.settings
        x = self.forward(logE, nu, record=True)
        L = self.losses(x, targets)
        _, _, gm, gl = self.solver.backward(2.0 * (x - targets), None, st.adjoint_iterations, st.adjoint_rho)
        mu, lam, dmu, dlam = self._materials(logE, nu)
        gm = gm.astype(np.float64)
        gl = gl.astype(np.float64)
        M = len(self.batch.meshes)
        g_logE = np.bincount(self.tet_mesh, weights=gm * mu + gl * lam, minlength=M)
        g_nu = np.bincount(self.tet_mesh, weights=gm * dmu + gl * dlam, minlength=M)
        return L, g_logE, g_nu

    def fd_grad(self, logE, nu, targets, which, eps=1e-4):
        """Central finite differences of every mesh's loss w.r.t. its log E (which='logE', step eps)
        or nu (which='nu', step eps * nu): two batched forwards."""
        logE = np.asarray(logE, np.float64)
        nu = np.asarray(nu, np.float64)
        if which == "logE":
            d = np.full_like(logE, eps)
            Lp = self.losses(self.forward(logE + d, nu), targets)
            Lm = self.losses(self.forward(logE - d, nu), targets)
        else:
            d = eps * nu
            Lp = self.losses(self.forward(logE, nu + d), targets)
            Lm = self.losses(self.forward(logE, nu - d), targets)
        return (Lp - Lm) / (2.0 * d)


NU_SCALE = 0.1  # nu is optimised as nu / NU_SCALE, so both coordinates move on similar scales


def identify(problem, targets, logE0, nu0, outer=50, nu_bounds=(0.05, 0.48), E_bounds=(5e3, 2e6), radius0=(1.0, 0.5),
             armijo=1e-4, fd_after=2, fd_step=1e-3, converged=1e-7, stall_window=5, stall_gain=0.1, trace=None):
    """Per-mesh trust-region descent on z = (log E, nu / NU_SCALE).

    Every mesh keeps its own trust radius (per coordinate, initially radius0).  Each outer
    iteration evaluates every mesh's trial point in one batched forward + adjoint; a mesh whose loss
    falls by the Armijo condition accepts the trial and widens its radius, the others halve it.
    Steps come from one of two models per mesh:
    * the adjoint's gradient with a 2x2 BFGS inverse-Hessian estimate;
    * once a mesh is on finite differences, a Levenberg-Marquardt step from the Jacobian J of its
      final positions with respect to z, taken by central differences (step fd_step) of the batched
      forward: (J^T J + m diag(J^T J)) d = -J^T r with r the positions minus the targets, the loss's
      gradient being 2 J^T r; m falls by 3 after an accepted step and grows by 4 after a rejected
      one.  The loss is a sum of squared residuals, so J^T J is its Gauss-Newton Hessian, which
      follows a long, curved (log E, nu) valley where a quasi-Newton estimate from two gradients
      crawls.  The four forwards of J are the ones the finite-difference gradient needs anyway; they
      run only while some mesh needs them, all meshes in each.
    The adjoint differentiates each step as converged; on stiff, nearly incompressible meshes the
    forward's fixed iteration count leaves the step far from converged, so that gradient can point
    away from descent.  A mesh whose trial has been rejected fd_after times in a row, while its loss
    is still above `converged` times its initial loss (below that, rejections come from FP32 noise
    in the loss), therefore switches to finite differences for good.  The same switch happens when a
    mesh's last stall_window accepted steps together lowered its loss by less than stall_gain of it:
    steps that are accepted but barely help also mark a gradient that does not point downhill.  nu
    is kept inside nu_bounds and E inside E_bounds (the batched configuration draws E from [1e4,
    1e6]; beyond it a very stiff beam barely moves, and the flat loss there holds a descent back).

    `problem` provides forward(logE, nu) -> final positions (N, 3), which it also leaves in
    problem.last_x, losses(x, targets) -> per-mesh losses, loss_and_grad(logE, nu, targets) (one
    forward, then the adjoint) and batch.vert_offsets.

    Returns (logE, nu, history of the total loss at the accepted points, per-mesh final losses, info)
    with info = dict(fd_meshes, forwards, forward_backwards).  A list passed as `trace` receives,
    per outer iteration, a dict of per-mesh arrays: z, loss, trial loss, accepted, radius, use_fd."""
    M = len(problem.batch.meshes)
    offs = np.asarray(problem.batch.vert_offsets)
    z = np.stack([np.asarray(logE0, np.float64), np.asarray(nu0, np.float64) / NU_SCALE], axis=1)
    lo = np.array([np.log(E_bounds[0]), nu_bounds[0] / NU_SCALE])
    hi = np.array([np.log(E_bounds[1]), nu_bounds[1] / NU_SCALE])
    z = np.clip(z, lo, hi)
    counts = {"forwards": 0, "forward_backwards": 0}

    def evaluate(zz):
        counts["forward_backwards"] += 1
        L, gE, gN = problem.loss_and_grad(zz[:, 0], zz[:, 1] * NU_SCALE, targets)
        return L, np.stack([gE, gN * NU_SCALE], axis=1), np.array(problem.last_x, np.float64, copy=True)

    def per_mesh(a):
        """Sums of a per-vertex quantity over each mesh's vertices."""
        return np.add.reduceat(a, offs[:-1])

    def gauss_newton(zz, xx):
        """J^T J (M, 2, 2) and J^T r (M, 2) of every mesh at zz, whose positions are xx, from central
        differences of the batched forward (four forwards)."""
        J = []
        for c, h in ((0, fd_step), (1, fd_step / NU_SCALE)):
            xs = []
            for sign in (1.0, -1.0):
                zt = zz.copy()
                zt[:, c] += sign * h
                counts["forwards"] += 1
                xs.append(np.asarray(problem.forward(zt[:, 0], zt[:, 1] * NU_SCALE), np.float64))
            J.append((xs[0] - xs[1]) / (2.0 * h))
        r = xx - targets
        A = np.empty((M, 2, 2))
        b = np.empty((M, 2))
        for i in range(2):
            b[:, i] = per_mesh(np.sum(J[i] * r, axis=1))
            for k in range(i, 2):
                A[:, i, k] = A[:, k, i] = per_mesh(np.sum(J[i] * J[k], axis=1))
        return A, b

    L, g, X = evaluate(z)
    L0 = L.copy()
    hist = [float(L.sum())]
    radius = np.tile(np.asarray(radius0, np.float64), (M, 1))
    Hinv = np.zeros((M, 2, 2))
    rejects = np.zeros(M, int)
    use_fd = np.zeros(M, bool)
    damping = np.full(M, 1e-3)  # Levenberg-Marquardt parameter of the finite-difference meshes
    accepted_losses = [[float(L[m])] for m in range(M)]  # loss after each accepted step

    def reset(m):
        Hinv[m] = np.eye(2) * (radius[m].min() / max(np.abs(g[m]).max(), 1e-300))

    def bfgs(m, s_, y_):
        sy = float(s_ @ y_)
        if sy > 1e-12 * np.linalg.norm(s_) * np.linalg.norm(y_):
            rho = 1.0 / sy
            V = np.eye(2) - rho * np.outer(s_, y_)
            Hinv[m] = V @ Hinv[m] @ V.T + rho * np.outer(s_, s_)

    for m in range(M):
        reset(m)
    for _ in range(outer):
        d = -np.einsum("mij,mj->mi", Hinv, g)
        if use_fd.any():
            A, b = gauss_newton(z, X)
            for m in np.flatnonzero(use_fd):
                g[m] = 2.0 * b[m]
                Am = A[m] + damping[m] * np.diag(np.diag(A[m])) + 1e-300 * np.eye(2)
                try:
                    d[m] = -np.linalg.solve(Am, b[m])
                except np.linalg.LinAlgError:
                    d[m] = -b[m] * radius[m].min() / max(np.abs(b[m]).max(), 1e-300)
        for m in range(M):
            if g[m] @ d[m] >= 0.0:  # not a descent direction: restart from a scaled gradient step
                reset(m)
                d[m] = -Hinv[m] @ g[m]
        d *= np.minimum(1.0, np.min(radius / np.maximum(np.abs(d), 1e-300), axis=1))[:, None]
        trial = np.clip(z + d, lo, hi)
        Lt, gt, Xt = evaluate(trial)
        step = trial - z
        ok = Lt <= L + armijo * np.einsum("mi,mi->m", g, step)
        for m in range(M):
            if not ok[m]:
                radius[m] *= 0.5
                rejects[m] += 1
                if use_fd[m]:
                    damping[m] *= 4.0
                elif rejects[m] >= fd_after and L[m] > converged * L0[m]:
                    use_fd[m] = True
                continue
            rejects[m] = 0
            radius[m] = np.minimum(2.0 * radius[m], 4.0 * np.asarray(radius0))
            if use_fd[m]:
                damping[m] = max(damping[m] / 3.0, 1e-12)
            else:
                bfgs(m, trial[m] - z[m], gt[m] - g[m])
                g[m] = gt[m]
            z[m], L[m] = trial[m], Lt[m]
            X[offs[m]:offs[m + 1]] = Xt[offs[m]:offs[m + 1]]
            hist_m = accepted_losses[m]
            hist_m.append(float(Lt[m]))
            if (not use_fd[m] and len(hist_m) > stall_window and L[m] > converged * L0[m]
                    and hist_m[-1 - stall_window] - hist_m[-1] < stall_gain * hist_m[-1 - stall_window]):
                use_fd[m] = True
        hist.append(float(L.sum()))
        if trace is not None:
            trace.append(dict(z=z.copy(), loss=L.copy(), trial_loss=np.asarray(Lt).copy(), accepted=ok.copy(),
                              radius=radius.copy(), use_fd=use_fd.copy()))
    info = dict(fd_meshes=int(use_fd.sum()), **counts)
    return z[:, 0], z[:, 1] * NU_SCALE, hist, L, info


def identify_adam(problem, targets, logE0, nu0, outer=50, lr_logE=0.15, lr_nu=0.01, nu_bounds=(0.05, 0.48)):
    """Adam on per-mesh (log E, nu); returns (logE, nu, history of total loss)."""
    logE = np.array(logE0, np.float64)
    nu = np.array(nu0, np.float64)
    mE = np.zeros_like(logE)
    vE = np.zeros_like(logE)
    mN = np.zeros_like(nu)
    vN = np.zeros_like(nu)
    b1, b2, eps = 0.9, 0.999, 1e-12
    hist = []
    for k in range(1, outer + 1):
        L, gE, gN = problem.loss_and_grad(logE, nu, targets)
        hist.append(float(L.sum()))
        mE = b1 * mE + (1 - b1) * gE
        vE = b2 * vE + (1 - b2) * gE * gE
        mN = b1 * mN + (1 - b1) * gN
        vN = b2 * vN + (1 - b2) * gN * gN
        logE -= lr_logE * (mE / (1 - b1 ** k)) / (np.sqrt(vE / (1 - b2 ** k)) + eps)
        nu -= lr_nu * (mN / (1 - b1 ** k)) / (np.sqrt(vN / (1 - b2 ** k)) + eps)
        nu = np.clip(nu, *nu_bounds)
    return logE, nu, hist
