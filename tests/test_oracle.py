"""The oracle itself: literal vs closed-form element blocks, finite differences of the energy,
precision and threading invariants, and the committed regression fixtures."""
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from vbd_tetmesh_b200 import meshgen

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def psi(F, mu, lam):
    J = np.linalg.det(F)
    return 0.5 * mu * (np.sum(F * F) - 3.0) - mu * (J - 1.0) + 0.5 * lam * (J - 1.0) ** 2


def random_element(rng):
    Dm = np.eye(3) * 0.05 + rng.normal(0, 0.01, (3, 3))
    Dinv = np.linalg.inv(Dm)
    F = np.eye(3) + rng.normal(0, 0.15, (3, 3))
    return F, Dinv, abs(np.linalg.det(Dm)) / 6.0


@pytest.mark.parametrize("n", [0, 1, 2, 3])
def test_closed_form_block_matches_literal_12x12(n):
    rng = np.random.default_rng(10 + n)
    for _ in range(50):
        F, Dinv, V = random_element(rng)
        mu, lam = 3.8e4, 5.7e4
        H_lit, g_lit = po.tet_block(F, Dinv, mu, lam, V, n, mode=po.LITERAL, precision=64)
        H_full, g_full = po.tet_block(F, Dinv, mu, lam, V, n, mode=po.LITERAL_FULL12, precision=64)
        H_cf, g_cf = po.tet_block(F, Dinv, mu, lam, V, n, mode=po.CLOSED, precision=64)
        np.testing.assert_array_equal(H_lit, H_full)
        scale = np.abs(H_lit).max()
        assert np.abs(H_lit - H_cf).max() <= 1e-12 * scale
        assert np.abs(g_lit - g_cf).max() <= 1e-12 * np.abs(g_lit).max()


def test_gradient_and_hessian_block_by_finite_differences():
    rng = np.random.default_rng(3)
    mu, lam = 3.8e4, 5.7e4
    for trial in range(10):
        Dm = np.eye(3) * 0.05 + rng.normal(0, 0.01, (3, 3))
        Dinv = np.linalg.inv(Dm)
        X = np.concatenate([np.zeros((1, 3)), Dm.T]) + rng.normal(0, 0.004, (4, 3))
        V = abs(np.linalg.det(Dm)) / 6.0

        def energy(Xc):
            Ds = np.stack([Xc[k] - Xc[0] for k in (1, 2, 3)], axis=1)
            return V * psi(Ds @ Dinv, mu, lam)

        Ds = np.stack([X[k] - X[0] for k in (1, 2, 3)], axis=1)
        F = Ds @ Dinv
        n = trial % 4
        H, g = po.tet_block(F, Dinv, mu, lam, V, n, mode=po.LITERAL, precision=64)
        eps = 1e-7
        g_fd = np.zeros(3)
        H_fd = np.zeros((3, 3))
        for c in range(3):
            Xp, Xm = X.copy(), X.copy()
            Xp[n, c] += eps
            Xm[n, c] -= eps
            g_fd[c] = (energy(Xp) - energy(Xm)) / (2 * eps)
            Hp, gp = po.tet_block(np.stack([Xp[k] - Xp[0] for k in (1, 2, 3)], 1) @ Dinv, Dinv, mu, lam, V, n,
                                  precision=64)
            Hm, gm = po.tet_block(np.stack([Xm[k] - Xm[0] for k in (1, 2, 3)], 1) @ Dinv, Dinv, mu, lam, V, n,
                                  precision=64)
            H_fd[:, c] = (gp - gm) / (2 * eps)
        np.testing.assert_allclose(g, g_fd, rtol=1e-5, atol=1e-6 * np.abs(g).max())
        np.testing.assert_allclose(H, H_fd, rtol=1e-5, atol=1e-6 * np.abs(H).max())


def _cof(A):
    """Cofactor matrix: cof(A) = det(A) A^-T, columns of cof([a b c]) = b x c, c x a, a x b."""
    return np.stack([np.cross(A[:, 1], A[:, 2]), np.cross(A[:, 2], A[:, 0]), np.cross(A[:, 0], A[:, 1])], axis=1)


@pytest.mark.parametrize("n", [0, 1, 2, 3])
def test_factored_record_identities(n):
    """The factored incidence records (layouts 3 and 4) rest on: F q_n = D s with s = M q_n,
    cof(F) q_n = cof(D) w with w = cof(M) q_n, J = det D det M, |q_n|^2 = -(s0 + s1 + s2), and (layout
    4, which stores no det M) det M = s . w / |q_n|^2.  M holds the other three vertices' rows of
    Q = Ps Dm^-1 in local order, D their positions minus vertex n's.  The element block built from
    them matches the oracle's closed form (Energy.cpp:90-158 restated) in FP64."""
    rng = np.random.default_rng(200 + n)
    mu, lam = 3.8e4, 5.7e4
    for _ in range(50):
        Dm = np.eye(3) * 0.05 + rng.normal(0, 0.01, (3, 3))
        Dinv = np.linalg.inv(Dm)
        X = np.concatenate([np.zeros((1, 3)), Dm.T]) + rng.normal(0, 0.004, (4, 3))
        V = abs(np.linalg.det(Dm)) / 6.0
        Q = np.concatenate([-Dinv.sum(axis=0, keepdims=True), Dinv])  # rows q_0 .. q_3
        others = [k for k in range(4) if k != n]
        M = Q[others]
        qn = Q[n]
        D = np.stack([X[k] - X[n] for k in others], axis=1)
        F = np.stack([X[k] - X[0] for k in (1, 2, 3)], axis=1) @ Dinv
        s, w = M @ qn, _cof(M) @ qn
        np.testing.assert_allclose(D @ M, F, rtol=0, atol=1e-12 * np.abs(F).max())
        np.testing.assert_allclose(F @ qn, D @ s, rtol=1e-12, atol=1e-12 * np.abs(F @ qn).max())
        np.testing.assert_allclose(_cof(F) @ qn, _cof(D) @ w, rtol=1e-11, atol=1e-11 * np.abs(_cof(F) @ qn).max())
        detM = np.linalg.det(M)
        assert abs(np.linalg.det(F) - np.linalg.det(D) * detM) <= 1e-12 * abs(np.linalg.det(F))
        qq = qn @ qn
        assert abs(-s.sum() - qq) <= 1e-12 * qq
        assert abs(s @ w / -s.sum() - detM) <= 1e-12 * abs(detM)
        # the kernel's element block from (D, s, w, det M, V mu, V lambda)
        Fq, Cq, J = D @ s, _cof(D) @ w, np.linalg.det(D) * detM
        a, b = V * mu, V * lam
        g = a * (Fq - Cq) + b * (J - 1.0) * Cq
        H = a * qq * np.eye(3) + b * np.outer(Cq, Cq)
        H_cf, g_cf = po.tet_block(F, Dinv, mu, lam, V, n, mode=po.CLOSED, precision=64)
        assert np.abs(H - H_cf).max() <= 1e-11 * np.abs(H_cf).max()
        assert np.abs(g - g_cf).max() <= 1e-11 * np.abs(g_cf).max()


def test_packed_id_bit_layout():
    """Layout 4 packs the other three vertex ids into 64 bits, 21 bits each (nb0 in bits 0-20, nb1
    in 21-41, nb2 in 42-62), written as two 32-bit words; this restates the kernels' encode
    (k_pack_factored) and decode (load of a packed record: a funnel shift for nb1) on ids up to
    2^21 - 1."""
    rng = np.random.default_rng(5)
    ids = np.concatenate([rng.integers(0, 1 << 21, (1000, 3)), [[0, 0, 0], [(1 << 21) - 1] * 3,
                                                                [(1 << 21) - 1, 0, (1 << 21) - 1]]]).astype(np.uint64)
    m32 = np.uint64(0xFFFFFFFF)
    lo = (ids[:, 0] | (ids[:, 1] << np.uint64(21))) & m32
    hi = ((ids[:, 1] >> np.uint64(11)) | (ids[:, 2] << np.uint64(10))) & m32
    mask = np.uint64((1 << 21) - 1)
    funnel = ((hi << np.uint64(32)) | lo) >> np.uint64(21)  # __funnelshift_r(lo, hi, 21), low 32 bits
    dec = np.stack([lo & mask, (funnel & m32) & mask, (hi >> np.uint64(10)) & mask], axis=1)
    np.testing.assert_array_equal(dec, ids)
    assert np.all(hi < np.uint64(1 << 31))  # bit 63 stays clear


def test_threaded_oracle_is_bit_identical_to_serial():
    m = meshgen.jittered_block(6, 5, 4, seed=1, per_tet_sigma=0.2)
    s = meshgen.BEAM_SETTINGS
    a = po.simulate(m, 3, s["dt"], 10, s["gravity"], True, 0.9, threads=1)
    b = po.simulate(m, 3, s["dt"], 10, s["gravity"], True, 0.9, threads=4)
    np.testing.assert_array_equal(a["x"], b["x"])
    np.testing.assert_array_equal(a["v"], b["v"])


def test_f32_oracle_close_to_f64():
    m = meshgen.beam()
    s = meshgen.BEAM_SETTINGS
    a = po.simulate(m, 10, s["dt"], s["iterations"], s["gravity"], True, s["rho"], precision=32)
    b = po.simulate(m, 10, s["dt"], s["iterations"], s["gravity"], True, s["rho"], precision=64)
    assert np.abs(a["x"] - b["x"]).max() / m.bbox_diag() < 2e-6


def test_oracle_matches_committed_fixtures():
    g = np.load(os.path.join(GOLDEN, "beam_oracle.npz"))
    m = meshgen.beam()
    s = meshgen.BEAM_SETTINGS
    for prec in (32, 64):
        for steps in (1, 10):
            r = po.simulate(m, steps, s["dt"], s["iterations"], s["gravity"], True, s["rho"], precision=prec)
            np.testing.assert_array_equal(r["x"], g[f"x_f{prec}_s{steps}"])
            np.testing.assert_array_equal(r["v"], g[f"v_f{prec}_s{steps}"])


def test_pinned_vertices_never_move_and_beam_sags():
    m = meshgen.beam()
    s = meshgen.BEAM_SETTINGS
    r = po.simulate(m, 10, s["dt"], s["iterations"], s["gravity"], True, s["rho"])
    fx = m.fixed.astype(bool)
    np.testing.assert_array_equal(r["x"][fx], m.x[fx].astype(np.float64))
    assert r["x"][~fx, 1].min() < -0.05


def test_energy_history_length():
    m = meshgen.beam(4, 2, 2)
    r = po.simulate(m, 2, 1 / 60, 20, use_acceleration=True, rho=0.9, energy_history=True)
    assert r["ehist"].shape == (2 * 2,)
    assert np.all(np.isfinite(r["ehist"]))
