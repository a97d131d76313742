"""VBD_OPT_SEMANTICS = 1: the reference GPU wrapper's semantics (VBD_GPU_Solver, VBD_GPU_Wrapper.cu
and VBD_DeviceMath.cuh) on this project's kernels.

Against the outputs of the reference's own GPU kernels (tests/golden/wrapper_ref.npz): bit-identical,
for single solveVBD calls and for frames of main.cpp's loop (whose predictor and velocity update
the reference runs on the host; the GPU predictor rounds y = x + h v the same way, without a fused
multiply-add).  Also within 1e-5 of the bounding-box diagonal of the oracle's restatement (mode
WRAPPER), and, where the reference library is built, bit-identical to the reference's kernels live."""
import os

import numpy as np
import pytest

from helpers import rel_err
from oracle import pyoracle as po
from vbd_tetmesh_b200 import VBDError, _capi, build_batch_solver, build_solver, meshgen

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "wrapper_ref.npz")
POS_TOL = 1e-5


def wrapper_frames(m, dt, iters, rho, frames, layout=0):
    s = build_solver(m, layout=layout)
    s.set_option(_capi.OPT_SEMANTICS, 1)
    s.set_velocities(np.zeros_like(m.x))
    for _ in range(frames):
        s.step(dt, iters, (0.0, -9.8, 0.0), True, rho)
    out = dict(x=s.get_positions(), v=s.get_velocities(), status=s.status())
    s.close()
    return out


CASES = {"beam": (lambda: meshgen.beam(), 1.0 / 60.0, 20, 0.95),
         "cube6": (lambda: meshgen.cube(6, E=1e6, nu=0.4, seed=5), 1.0 / 120.0, 50, 0.9)}


@pytest.mark.parametrize("layout", [0, 1, 3])
@pytest.mark.parametrize("case,frames", [("beam", 1), ("beam", 5), ("cube6", 1), ("cube6", 3)])
def test_frames_match_reference_gpu(gpu_device, case, frames, layout):
    gold = np.load(GOLDEN)
    make, dt, iters, rho = CASES[case]
    m = make()
    g = wrapper_frames(m, dt, iters, rho, frames, layout)
    ref = gold[f"{case}/x_f{frames}"]
    err = rel_err(g["x"], ref, m)
    print(f"{case} frames={frames} layout={layout}: vs reference GPU {err:.2e}, "
          f"bit-identical={np.array_equal(g['x'], ref)}")
    assert err < POS_TOL
    assert g["status"] == (0, False)
    np.testing.assert_array_equal(g["x"], ref)
    np.testing.assert_array_equal(g["v"], gold[f"{case}/v_f{frames}"])


@pytest.mark.parametrize("accel", [0, 1])
def test_solve_bit_identical_to_reference_gpu(gpu_device, accel):
    gold = np.load(GOLDEN)
    m = meshgen.jittered_block(6, 4, 5, seed=3)
    s = build_solver(m, layout=0)
    s.set_option(_capi.OPT_SEMANTICS, 1)
    s.update_inertia_from_cpu(gold["solve/y"])
    s.solve_vbd(30, 3600.0, bool(accel), 0.9, _capi.INIT_FROM_INERTIA)
    x = s.get_positions()
    s.close()
    np.testing.assert_array_equal(x, gold[f"solve/x_accel{accel}"])


def test_matches_wrapper_oracle(gpu_device):
    m = meshgen.jittered_block(8, 4, 4, seed=21, per_tet_sigma=0.3)
    g = wrapper_frames(m, 1.0 / 60.0, 15, 0.9, 4)
    o = po.simulate(m, 4, 1.0 / 60.0, 15, (0.0, -9.8, 0.0), True, 0.9, precision=32, mode=po.WRAPPER,
                    v0=np.zeros_like(m.x))
    o64 = po.simulate(m, 4, 1.0 / 60.0, 15, (0.0, -9.8, 0.0), True, 0.9, precision=64, mode=po.WRAPPER,
                      v0=np.zeros_like(m.x))
    e32, e64 = rel_err(g["x"], o["x"], m), rel_err(g["x"], o64["x"], m)
    print(f"per-tet materials, 4 frames: vs wrapper oracle32 {e32:.2e}, vs oracle64 {e64:.2e}")
    assert e32 < POS_TOL


@pytest.mark.skipif(not po.ref_gpu_available(), reason="oracle/_ref/libvbdref_gpu.so not built")
def test_cube_solve_bit_identical_to_live_reference(gpu_device):
    m = meshgen.cube(16)
    rng = np.random.default_rng(4)
    y = (m.x + 1e-3 * rng.normal(size=m.x.shape)).astype(np.float32)
    y[m.fixed == 1] = m.x[m.fixed == 1]
    h = po.RefGpuHandle(m, iterations=50, rho=0.9)
    h.set_inertia(y)
    h.solve(50, 14400.0, True, 0.9)
    xr = h.positions()
    h.close()
    s = build_solver(m, layout=0)
    s.set_option(_capi.OPT_SEMANTICS, 1)
    s.update_inertia_from_cpu(y)
    s.solve_vbd(50, 14400.0, True, 0.9, _capi.INIT_FROM_INERTIA)
    x = s.get_positions()
    s.close()
    np.testing.assert_array_equal(x, xr)


def test_batched_wrapper_semantics_bit_identical_to_per_mesh(gpu_device):
    meshes = meshgen.batched_blocks(num_meshes=5, lo=2, hi=6, seed=9)
    b = meshgen.concat(meshes)
    s = build_batch_solver(b)
    s.set_option(_capi.OPT_SEMANTICS, 1)
    for _ in range(3):
        s.step(1 / 60, 20, (0.0, -9.8, 0.0), True, 0.9)
    xs = b.split(s.get_positions())
    s.close()
    for m, x in zip(meshes, xs):
        p = build_solver(m)
        p.set_option(_capi.OPT_SEMANTICS, 1)
        for _ in range(3):
            p.step(1 / 60, 20, (0.0, -9.8, 0.0), True, 0.9)
        np.testing.assert_array_equal(x, p.get_positions())
        p.close()


def test_semantics_option_rules(gpu_device):
    m = meshgen.jittered_block(3, 2, 2, seed=1)
    s = build_solver(m)
    assert s.get_option(_capi.OPT_SEMANTICS) == 0
    with pytest.raises(VBDError):
        s.set_option(_capi.OPT_SEMANTICS, 2)
    s.set_option(_capi.OPT_PERSISTENT, 1)
    with pytest.raises(VBDError):
        s.set_option(_capi.OPT_SEMANTICS, 1)
    s.set_option(_capi.OPT_PERSISTENT, 0)
    s.set_option(_capi.OPT_SEMANTICS, 1)
    with pytest.raises(VBDError):
        s.set_option(_capi.OPT_PERSISTENT, 1)
    with pytest.raises(VBDError):
        s.record(2)
    s.set_option(_capi.OPT_SEMANTICS, 0)
    s.record(2)
    with pytest.raises(VBDError):
        s.set_option(_capi.OPT_SEMANTICS, 1)
    s.record(0)
    s.close()
