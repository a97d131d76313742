"""Greedy colouring: the library's C++ colouring is bit-exact with the oracle's restatement of
GraphColoring::colorVertices (GraphColoring.cpp:28-66) and yields independent colour classes."""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from vbd_tetmesh_b200 import color_vertices, meshgen

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "colouring.json")


def independent(colour_of, tets):
    c = colour_of[tets]
    for a in range(4):
        for b in range(a):
            if np.any(c[:, a] == c[:, b]):
                return False
    return True


def random_soup(n, t, seed):
    rng = np.random.default_rng(seed)
    return np.stack([rng.choice(n, 4, replace=False) for _ in range(t)]).astype(np.int32)


CASES = {
    "beam": lambda: (meshgen.beam().num_verts, meshgen.beam().tets),
    "block_6x4x5": lambda: (lambda m: (m.num_verts, m.tets))(meshgen.jittered_block(6, 4, 5, seed=3)),
    "block_1x1x1": lambda: (lambda m: (m.num_verts, m.tets))(meshgen.jittered_block(1, 1, 1)),
    "soup_200_600": lambda: (200, random_soup(200, 600, 0)),
    "soup_50_400": lambda: (50, random_soup(50, 400, 1)),
    "isolated_vertices": lambda: (10, np.array([[0, 1, 2, 3], [2, 3, 4, 5]], np.int32)),
    "no_tets": lambda: (5, np.zeros((0, 4), np.int32)),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_colouring_bit_exact_with_oracle(case):
    n, tets = CASES[case]()
    c_lib, offs, verts = color_vertices(n, tets)
    c_orc, nc = po.color_vertices(n, tets)
    assert nc == len(offs) - 1
    np.testing.assert_array_equal(c_lib, c_orc)
    assert independent(c_lib, tets)
    # groups in ascending vertex id, partitioning the vertices
    for c in range(nc):
        g = verts[offs[c]:offs[c + 1]]
        assert np.all(np.diff(g) > 0) and np.all(c_lib[g] == c)
    assert offs[-1] == n


def cube_colouring():
    m = meshgen.cube(64)
    return m, color_vertices(m.num_verts, m.tets)


def test_cube_colouring_golden_and_oracle():
    m, (c_lib, offs, verts) = cube_colouring()
    assert (m.num_verts, m.num_tets) == (274625, 1572864)
    sizes = np.diff(offs).tolist()
    assert sizes == [35937, 51520, 39813, 48895, 35925, 28263, 17136, 17136]
    c_orc, nc = po.color_vertices(m.num_verts, m.tets)
    np.testing.assert_array_equal(c_lib, c_orc)
    assert independent(c_lib, m.tets)
    golden = json.load(open(GOLDEN))
    assert hashlib.sha256(c_lib.tobytes()).hexdigest() == golden["cube64"]["sha256"]


def test_config_meshes_colour_counts():
    for m, expect in ((meshgen.beam(), 8), (meshgen.beam(32, 8, 8), 8)):
        _, offs, _ = color_vertices(m.num_verts, m.tets)
        assert len(offs) - 1 == expect
