"""Accuracy of the factored element records (layouts 3 and 4) on well-shaped, anisotropic and sliver
meshes: the FP32 det M they use against FP64 (vbd_factored_record_error, host only), which is what
vbd_solver_init's automatic layout choice tests.  Both factored layouts form the element block from
det M: layout 3 stores it, layout 4 derives it as s.w / |q_n|^2, where |q_n|^2 = -(s_0 + s_1 + s_2)
cancels when a vertex's gradient row is small next to the others."""
import numpy as np

from vbd_tetmesh_b200 import meshgen, precompute_tets
from vbd_tetmesh_b200.solver import factored_record_error

TOL = 1e-5  # the automatic layout choice's bar


def _err(m):
    dm, _ = precompute_tets(m.rest, m.tets)
    return factored_record_error(dm)[:2]


def _keeps_packed(m):
    """vbd_solver_init's automatic choice: the packed layout 4 unless its derived det M is worse than
    both 1e-5 and 4 times the stored one's error on more than 0.1% of the incidences."""
    dm, _ = precompute_tets(m.rest, m.tets)
    return factored_record_error(dm)[2] <= 1e-3


def flattened(factor, seed=4):
    m = meshgen.jittered_block(8, 8, 8, cell=0.05, jitter=0.1, seed=seed)
    m.rest = m.rest.copy()
    m.rest[:, 2] /= factor
    m.x = m.rest.copy()
    return m


def test_well_shaped_meshes_keep_the_packed_layout():
    for m in (meshgen.cube(24), meshgen.cube(64), meshgen.beam(32, 8, 8)):
        e3, e4 = _err(m)
        assert e4 < TOL and e3 < TOL, (m.dims, e3, e4)
        assert _keeps_packed(m)


def test_anisotropic_mesh_needs_the_stored_det():
    e3, e4 = _err(flattened(1000))
    assert e4 > TOL      # |q_n|^2 cancels: about 1e-4
    assert e3 < 1e-6     # the stored det M stays accurate
    assert not _keeps_packed(flattened(1000))


def test_sliver_tets_limit_both_factored_layouts():
    """Near-sliver tets carry the FP32 conditioning error of Dm^-1 in both factored layouts; on a
    mesh made of them (+-0.49-cell jitter) layout 4 loses accuracy on enough incidences for the
    automatic choice to take layout 3.  The batched configuration's +-0.25-cell jitter makes only
    isolated thin tets (a few incidences in a hundred thousand), so that batch keeps layout 4: its
    positions after 60 steps are as close to FP64 with layout 4 as with layout 3
    (tests/test_gpu_parity_headline.py)."""
    m = meshgen.jittered_block(8, 8, 8, cell=0.05, jitter=0.49, seed=3)
    e3, e4 = _err(m)
    assert e3 > TOL and e4 > TOL
    assert not _keeps_packed(m)
    dm = np.concatenate([precompute_tets(m.rest, m.tets)[0] for m in meshgen.batched_blocks(64)])
    e3, e4, frac = factored_record_error(dm)
    assert e4 > TOL and 0.0 < frac < 1e-4


def test_error_matches_a_numpy_restatement():
    """The estimator's layout-3 figure equals an independent FP32 restatement of the stored det M."""
    m = flattened(100)
    dm, _ = precompute_tets(m.rest, m.tets)
    e3 = factored_record_error(dm)[0]
    D = dm.astype(np.float32)
    Q = np.concatenate([(-D[:, 0] - D[:, 1] - D[:, 2])[:, None], D], axis=1)
    worst = 0.0
    for n in range(4):
        M = Q[:, [k for k in range(4) if k != n]]
        c0 = (M[:, 1, [1, 2, 0]] * M[:, 2, [2, 0, 1]] - M[:, 1, [2, 0, 1]] * M[:, 2, [1, 2, 0]]).astype(np.float32)
        det32 = (M[:, 0, 0] * c0[:, 0] + M[:, 0, 1] * c0[:, 1] + M[:, 0, 2] * c0[:, 2]).astype(np.float32)
        exact = np.linalg.det(M.astype(np.float64))
        worst = max(worst, float(np.max(np.abs(det32 / exact - 1.0))))
    assert abs(e3 - worst) <= 0.5 * worst + 1e-7
