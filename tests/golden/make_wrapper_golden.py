"""Generates tests/golden/wrapper_ref.npz: outputs of the reference's own GPU path
(VBD::VBD_GPU_Solver from VBD_GPU_Wrapper.cu, built by `make -C oracle refgpu` into
oracle/_ref/libvbdref_gpu.so) on small meshes.  They pin the wrapper-semantics restatement of the
oracle (mode WRAPPER) and this project's VBD_OPT_SEMANTICS = 1 path.

Runs on a machine with a GPU and the built library:
    python tests/golden/make_wrapper_golden.py [output.npz]   (default: tests/golden/wrapper_ref.npz)

Cases (float32 arrays):
  beam/*   meshgen.beam(): main.cpp's GPU loop, dt 1/60, 1 substep, 20 iterations, rho 0.95,
           gravity (0, -9.8, 0); positions and velocities after 1 and 5 frames.
  cube6/*  meshgen.cube(6, E=1e6, nu=0.4, seed=5) (initial velocities dropped: main.cpp starts from
           rest), dt 1/120, 50 iterations, rho 0.9; after 1 and 3 frames.
  solve/*  meshgen.jittered_block(6, 4, 5, seed=3): one solveVBD of 30 iterations, rho 0.9, from the
           inertial target y = x + 0.02 sin(...) (seeded), 1/h^2 = 3600, with and without Chebyshev.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle as po  # noqa: E402
from vbd_tetmesh_b200 import meshgen  # noqa: E402


def frames(m, dt, iters, rho, counts):
    h = po.RefGpuHandle(m, dt=dt, iterations=iters, rho=rho)
    out = {}
    done = 0
    for c in counts:
        h.frame(c - done)
        done = c
        out[f"x_f{c}"] = h.positions()
        out[f"v_f{c}"] = h.velocities()
    h.close()
    return out


def solve_case():
    m = meshgen.jittered_block(6, 4, 5, seed=3)
    rng = np.random.default_rng(11)
    y = (m.x + 0.02 * np.sin(rng.uniform(0, 6.28, m.x.shape))).astype(np.float32)
    y[m.fixed == 1] = m.x[m.fixed == 1]
    out = {"y": y}
    for accel in (0, 1):
        h = po.RefGpuHandle(m)
        h.set_inertia(y)
        h.solve(30, 3600.0, bool(accel), 0.9)
        out[f"x_accel{accel}"] = h.positions()
        h.close()
    return out


def main():
    data = {}
    beam = meshgen.beam()
    for k, v in frames(beam, 1.0 / 60.0, 20, 0.95, (1, 5)).items():
        data[f"beam/{k}"] = v
    cube = meshgen.cube(6, E=1e6, nu=0.4, seed=5)
    cube.v[:] = 0.0
    for k, v in frames(cube, 1.0 / 120.0, 50, 0.9, (1, 3)).items():
        data[f"cube6/{k}"] = v
    for k, v in solve_case().items():
        data[f"solve/{k}"] = v
    path = sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "wrapper_ref.npz")
    np.savez_compressed(path, **data)
    print("wrote", path, {k: v.shape for k, v in data.items()})


if __name__ == "__main__":
    main()
