"""Config meshes have the sizes the benchmark configurations state."""
import numpy as np

from vbd_tetmesh_b200 import meshgen


def test_beam_sizes():
    m = meshgen.beam()
    assert (m.num_verts, m.num_tets, int(m.fixed.sum())) == (425, 1536, 25)


def test_diff_beam_sizes():
    m = meshgen.beam(32, 8, 8)
    assert (m.num_verts, m.num_tets) == (2673, 12288)


def test_cube_sizes_and_pins():
    m = meshgen.cube(64)
    assert (m.num_verts, m.num_tets, int(m.fixed.sum())) == (274625, 1572864, 4225)
    assert np.all(m.v[m.fixed.astype(bool)] == 0)
    assert 0.45 < float(m.v[~m.fixed.astype(bool)].std()) < 0.55


def test_kuhn_split_is_conforming_and_fills_cells():
    pos, tets, _ = meshgen.grid(3, 2, 2, 1.0)
    D = np.stack([pos[tets[:, k]] - pos[tets[:, 0]] for k in (1, 2, 3)], axis=2)
    vol = np.abs(np.linalg.det(D)) / 6.0
    assert np.allclose(vol, 1.0 / 6.0) and abs(vol.sum() - 12.0) < 1e-9
    faces = np.sort(np.concatenate([tets[:, [0, 1, 2]], tets[:, [0, 1, 3]], tets[:, [0, 2, 3]], tets[:, [1, 2, 3]]]),
                    axis=1)
    _, counts = np.unique(faces, axis=0, return_counts=True)
    assert counts.max() == 2
    assert (counts == 1).sum() == 2 * (3 * 2 + 3 * 2 + 2 * 2) * 2


def test_batched_config_sizes():
    ms = meshgen.batched_blocks()
    b = meshgen.concat(ms)
    assert len(ms) == 512
    assert 1.5e6 < b.num_verts < 1.9e6 and 7.5e6 < b.num_tets < 9.5e6
    dims = np.array([m.dims for m in ms])
    assert dims.min() >= 4 and dims.max() <= 24
    assert all(m.fixed.sum() > 0 for m in ms)
    E = np.array([m.meta["E"] for m in ms])
    assert 1e4 <= E.min() and E.max() <= 1e6
