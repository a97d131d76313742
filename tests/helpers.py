"""Shared helpers of the test suite (meshes, GPU runs, error measures)."""
import numpy as np

from vbd_tetmesh_b200 import build_solver, meshgen


def rel_err(a, b, mesh):
    """max |a - b| over all coordinates, divided by the mesh's bounding-box diagonal."""
    return float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max() / mesh.bbox_diag())


def gpu_simulate(mesh, steps, dt, iterations, gravity=(0.0, -9.8, 0.0), use_acceleration=True, rho=0.95,
                 substeps=1, lanes=None, layout=None, graph=None, device=0, options=None):
    s = build_solver(mesh, device=device, lanes=lanes, layout=layout, graph=graph)
    for k, v in (options or {}).items():
        s.set_option(k, v)
    try:
        l0 = s.kernel_launches()
        for _ in range(steps):
            s.step(dt, iterations, gravity, use_acceleration, rho, substeps)
        s.sync()
        launches = s.kernel_launches() - l0
        x = s.get_positions()
        v = s.get_velocities()
        h = dt / substeps
        ip = s.energy(0, h)
        sing, nonf = s.status()
        return dict(x=x, v=v, ip=ip, singular=sing, nonfinite=nonf, launches=launches)
    finally:
        s.close()


def small_block(seed=0, dims=(6, 4, 5), per_tet_sigma=0.2, pin="x0", E=1e5, nu=0.3, jitter=0.25):
    return meshgen.jittered_block(*dims, cell=0.05, jitter=jitter, E=E, nu=nu, seed=seed, pin_face=pin,
                                  per_tet_sigma=per_tet_sigma)
