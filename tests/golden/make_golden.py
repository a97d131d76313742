"""Regenerates the fixtures in tests/golden from the oracle (oracle/libvbd_oracle.so).

    python tests/golden/make_golden.py

colouring.json   sha256 of the greedy colour assignment (int32 array bytes) of the config meshes
beam_oracle.npz  oracle trajectories of the 16x4x4 beam (dt 1/60, 20 iterations, Chebyshev 0.95,
                 gravity -9.8 y): positions / velocities after 1 and 10 steps, FP32 and FP64
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import pyoracle as po  # noqa: E402
from vbd_tetmesh_b200 import meshgen  # noqa: E402


def main():
    out = {}
    for name, m in (("beam", meshgen.beam()), ("diffbeam", meshgen.beam(32, 8, 8)), ("cube64", meshgen.cube(64))):
        c, nc = po.color_vertices(m.num_verts, m.tets)
        out[name] = dict(sha256=hashlib.sha256(c.tobytes()).hexdigest(), colours=int(nc),
                         sizes=np.bincount(c).tolist())
    json.dump(out, open(os.path.join(HERE, "colouring.json"), "w"), indent=1)

    m = meshgen.beam()
    s = meshgen.BEAM_SETTINGS
    arrs = {}
    for prec in (32, 64):
        for steps in (1, 10):
            r = po.simulate(m, steps, s["dt"], s["iterations"], s["gravity"], True, s["rho"], precision=prec)
            arrs[f"x_f{prec}_s{steps}"] = r["x"]
            arrs[f"v_f{prec}_s{steps}"] = r["v"]
            arrs[f"ip_f{prec}_s{steps}"] = r["ip"]
    np.savez_compressed(os.path.join(HERE, "beam_oracle.npz"), **arrs)


if __name__ == "__main__":
    main()
