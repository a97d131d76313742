"""Pins the oracle to the reference's own code.

The reference's sources (TetMesh.h, VBD.cpp, Energy.cpp, GraphColoring.cpp, NeoHookean.cpp) compile
unchanged against this project's Eigen-API subset (`make -C oracle ref`, oracle/_ref/).  The oracle's
restatement must reproduce that build bit for bit: set-up products (colours, masses, rest volumes,
Dm^-1, V0) and positions / velocities after 1 and 10 steps.  The committed fixtures
(tests/golden/ref_trajectories.npz, from tests/golden/make_ref_golden.py) carry the check to machines
without the reference tree; where oracle/_ref is built, extra cases run live.  computeTotalEnergy is
compared with a tolerance: the reference takes J from a singular-value product (JacobiSVD), the oracle
from |det F|.
"""
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from vbd_tetmesh_b200 import meshgen

sys_path_golden = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys_path_golden_file = os.path.join(sys_path_golden, "ref_trajectories.npz")

import importlib.util  # noqa: E402

_spec = importlib.util.spec_from_file_location("make_ref_golden", os.path.join(sys_path_golden, "make_ref_golden.py"))
_mrg = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(_mrg)
CASES = _mrg.CASES
ENERGY_RTOL = 1e-4


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_bit_exact_with_reference_fixtures(name):
    g = np.load(sys_path_golden_file)
    make, dt, iters, accel, rho, sub = CASES[name]
    m = make()
    mass, trv, dm, v0 = po.mesh_setup(m.rest, m.tets, m.density, precision=32)
    col, _ = po.color_vertices(m.num_verts, m.tets)
    np.testing.assert_array_equal(col, g[f"{name}/colour_of"])
    np.testing.assert_array_equal(mass, g[f"{name}/mass"].astype(np.float64))
    np.testing.assert_array_equal(trv, g[f"{name}/tet_rest_vol"].astype(np.float64))
    np.testing.assert_array_equal(dm, g[f"{name}/dminv"].astype(np.float64))
    np.testing.assert_array_equal(v0, g[f"{name}/v0"].astype(np.float64))
    for steps in (1, 10):
        o = po.simulate(m, steps, dt, iters, (0.0, -9.8, 0.0), accel, rho, substeps=sub, precision=32,
                        energy_history=(steps == 10))
        np.testing.assert_array_equal(o["x"], g[f"{name}/x_s{steps}"].astype(np.float64))
        np.testing.assert_array_equal(o["v"], g[f"{name}/v_s{steps}"].astype(np.float64))
    eh = g[f"{name}/ehist"]
    np.testing.assert_allclose(o["ehist"][: len(eh)], eh, rtol=ENERGY_RTOL, atol=ENERGY_RTOL * np.abs(eh).max())


LIVE = {
    "block_seed11_accel": (lambda: meshgen.jittered_block(5, 5, 3, seed=11, E=8e4, nu=0.25), 1 / 60, 15, True, 0.8, 1),
    "block_pinned_y": (lambda: meshgen.jittered_block(4, 6, 4, seed=12, pin_face="y0"), 1 / 90, 10, True, 0.9, 3),
    "beam_32x8x8": (lambda: meshgen.beam(32, 8, 8), 1 / 60, 30, True, 0.95, 1),
}


@pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref not built (needs the reference tree)")
@pytest.mark.parametrize("name", sorted(LIVE))
def test_oracle_bit_exact_with_reference_live(name):
    make, dt, iters, accel, rho, sub = LIVE[name]
    m = make()
    r = po.RefHandle(m, dt, iters, (0.0, -9.8, 0.0), accel, rho, substeps=sub)
    r.step(3)
    x, v = r.state()
    o = po.simulate(m, 3, dt, iters, (0.0, -9.8, 0.0), accel, rho, substeps=sub, precision=32)
    np.testing.assert_array_equal(o["x"], x.astype(np.float64))
    np.testing.assert_array_equal(o["v"], v.astype(np.float64))
