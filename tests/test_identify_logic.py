"""Host logic of the material identification's optimiser (vbd_tetmesh_b200.material_id.identify)
on a stand-in problem without a GPU: each "mesh" has a quadratic loss in (log E, nu) around its
hidden parameters, the batched forward returns the parameters themselves, and one mesh's
implicit gradient is made to mislead the way an unconverged forward's does (barely downhill, mostly
across the valley), so its steps are rejected or stall."""
import numpy as np

from vbd_tetmesh_b200 import material_id as mid


class _Batch:
    def __init__(self, m):
        self.meshes = [None] * m
        self.vert_offsets = np.arange(m + 1)


class FakeProblem:
    def __init__(self, logE_true, nu_true, misleading=()):
        self.truth = np.stack([logE_true, nu_true], axis=1)
        self.batch = _Batch(len(logE_true))
        self.misleading = np.zeros(len(logE_true), bool)
        self.misleading[list(misleading)] = True
        self.forwards = 0

    def forward(self, logE, nu, record=False):
        self.forwards += 1
        self.last_x = np.stack([np.asarray(logE, np.float64), np.asarray(nu, np.float64) / mid.NU_SCALE], axis=1)
        return self.last_x

    def losses(self, x, targets):
        return np.sum((x - targets) ** 2, axis=1)

    def targets(self):
        return self.forward(self.truth[:, 0], self.truth[:, 1])

    def loss_and_grad(self, logE, nu, targets):
        x = self.forward(logE, nu)
        L = self.losses(x, targets)
        g = 2.0 * (x - targets)
        # the implicit gradient of an unconverged forward: still (barely) a descent direction, but
        # mostly across the valley
        gm = g[self.misleading]
        g[self.misleading] = 0.05 * gm + np.stack([-gm[:, 1], gm[:, 0]], axis=1)
        return L, g[:, 0], g[:, 1] / mid.NU_SCALE


def test_identify_recovers_parameters_and_switches_misled_mesh_to_finite_differences():
    logE_true = np.log(np.array([2e4, 3e5, 8e5, 5e4]))
    nu_true = np.array([0.25, 0.35, 0.44, 0.3])
    prob = FakeProblem(logE_true, nu_true, misleading=[2])
    t = prob.targets()
    trace = []
    logE, nu, hist, L, info = mid.identify(prob, t, np.full(4, np.log(1e5)), np.full(4, 0.3), outer=60, trace=trace)
    assert info["fd_meshes"] >= 1 and trace[-1]["use_fd"][2]
    np.testing.assert_allclose(np.exp(logE), np.exp(logE_true), rtol=1e-3)
    np.testing.assert_allclose(nu, nu_true, atol=1e-3)
    assert hist[-1] < 1e-6 * hist[0]
    # every accepted loss is no larger than the one before it (Armijo)
    losses = np.array([s["loss"] for s in trace])
    assert np.all(np.diff(losses, axis=0) <= 1e-12)


def test_identify_keeps_E_and_nu_inside_bounds():
    # a hidden E above the bound: the estimate stops at the bound instead of running off
    logE_true = np.log(np.array([5e7, 1e5]))
    nu_true = np.array([0.3, 0.49])
    prob = FakeProblem(logE_true, nu_true)
    logE, nu, hist, L, info = mid.identify(prob, prob.targets(), np.full(2, np.log(1e5)), np.full(2, 0.3), outer=40,
                                           E_bounds=(5e3, 2e6), nu_bounds=(0.05, 0.48))
    assert np.exp(logE[0]) <= 2e6 * (1 + 1e-12)
    assert np.isclose(np.exp(logE[0]), 2e6, rtol=1e-6)
    assert nu[1] <= 0.48 + 1e-12 and np.isclose(nu[1], 0.48, atol=1e-6)
