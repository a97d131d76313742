"""Regenerates tests/golden/ref_trajectories.npz from the reference's own sources.

    make -C oracle ref                       # reference sources + Eigen-API subset -> oracle/_ref/
    python tests/golden/make_ref_golden.py

For each case: the reference's set-up products (colours, masses, rest volumes, Dm^-1, V0) and its
positions / velocities after 1 and 10 VBDsolver::step calls (numThreads = 1), plus its
computeTotalEnergy history.  The oracle is checked against these arrays in tests/test_oracle_pin.py.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import pyoracle as po  # noqa: E402
from vbd_tetmesh_b200 import meshgen  # noqa: E402

CASES = {
    # name: (mesh factory, dt, iterations, use_acceleration, rho, substeps)
    "beam": (lambda: meshgen.beam(), 1 / 60, 20, True, 0.95, 1),
    "block_accel_off_sub2": (lambda: meshgen.jittered_block(6, 4, 5, seed=3, E=2e5, nu=0.35), 1 / 60, 12, False,
                             0.0, 2),
    "cube6_stiff": (lambda: meshgen.cube(6, seed=5), 1 / 120, 50, True, 0.9, 1),
}


def main():
    out = {}
    for name, (make, dt, iters, accel, rho, sub) in CASES.items():
        m = make()
        r = po.RefHandle(m, dt, iters, (0.0, -9.8, 0.0), accel, rho, substeps=sub, threads=1)
        su = r.setup()
        for k, v in su.items():
            if k != "ncolours":
                out[f"{name}/{k}"] = v
        r.step(1)
        out[f"{name}/x_s1"], out[f"{name}/v_s1"] = r.state()
        r.step(9)
        out[f"{name}/x_s10"], out[f"{name}/v_s10"] = r.state()
        out[f"{name}/ehist"] = r.energy_history()
        r.close()
    np.savez_compressed(os.path.join(HERE, "ref_trajectories.npz"), **out)


if __name__ == "__main__":
    main()
