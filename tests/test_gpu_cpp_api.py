"""The C++ drop-in surface on the GPU: tests/cpp/test_cpp_api runs the reference's two calling
patterns (VBDsolver::step, and the main.cpp loop over VBD_GPU_Solver) through include/vbd/*.h and
libvbd_b200; results are checked against the oracle."""
import dataclasses
import importlib.util
import os
import subprocess

import numpy as np
import pytest

from helpers import rel_err
from oracle import pyoracle as po
from vbd_tetmesh_b200 import meshgen

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CPP_DIR = os.path.join(ROOT, "tests", "cpp")
BIN = os.path.join(CPP_DIR, "test_cpp_api")
SIM_BIN = os.path.join(CPP_DIR, "test_simulate")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def run_cpp(m, iters, steps, dt, rho, tmp_path):
    if not os.path.exists(BIN):
        subprocess.run(["make", "-C", CPP_DIR], check=True, capture_output=True)
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        np.array([m.num_verts, m.num_tets, iters, steps], np.int32).tofile(f)
        np.array([m.density, m.mu[0], m.lam[0], dt, rho], np.float32).tofile(f)
        m.rest.astype(np.float32).tofile(f)
        m.tets.astype(np.int32).tofile(f)
        m.fixed.astype(np.uint8).tofile(f)
    out = tmp_path / "out.bin"
    obj = tmp_path / "mesh.obj"
    r = subprocess.run([BIN, str(inp), str(out), str(obj)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    raw = open(out, "rb").read()
    n3 = 3 * m.num_verts
    k = 4 * (3 * n3 + 1)
    f = np.frombuffer(raw[:k], np.float32)
    tail = np.frombuffer(raw[k:k + 8], np.int32)
    x3 = np.frombuffer(raw[k + 8:], np.float32)
    assert x3.size == n3
    return dict(x1=f[:n3].reshape(-1, 3), v1=f[n3:2 * n3].reshape(-1, 3), x2=f[2 * n3:3 * n3].reshape(-1, 3),
                energy=float(f[3 * n3]), nsurf=int(tail[0]), ncol=int(tail[1]), obj=obj, x3=x3.reshape(-1, 3))


def per_tet_flow_oracle(m, iters, steps, dt, rho):
    """test_cpp_api's flow 3 by the FP32 oracle: VBDsolver::step with per-tet materials mu (1 + t%5 / 8),
    lambda (1 + t%3 / 4), and mu of every even tet times 1.5 from step steps // 2 on."""
    t = np.arange(m.num_tets)
    mu = np.float32(m.mu[0]) * (np.float32(1.0) + np.float32(0.125) * (t % 5).astype(np.float32))
    lam = np.float32(m.lam[0]) * (np.float32(1.0) + np.float32(0.25) * (t % 3).astype(np.float32))
    mu2 = mu.copy()
    mu2[::2] *= np.float32(1.5)
    half = steps // 2
    a = po.simulate(dataclasses.replace(m, mu=mu, lam=lam), half, dt, iters, (0.0, -9.8, 0.0), True, rho, precision=32)
    b = po.simulate(dataclasses.replace(m, mu=mu2, lam=lam), steps - half, dt, iters, (0.0, -9.8, 0.0), True, rho,
                    precision=32, x0=a["x"], v0=a["v"])
    return b["x"]


def wrapper_flow_oracle(m, iters, steps, dt, rho):
    """The main.cpp loop: host predictor (float32, TetMesh.h:319-348), solveVBD from x = y with the
    GPU wrapper's semantics (VBD_GPU_Wrapper.cu:332-362) by the oracle, host velocity update
    (TetMesh.h:305-311)."""
    dt32 = np.float32(dt)
    dtsr = np.float32(1.0) / (dt32 * dt32)
    x = m.x.astype(np.float32).copy()
    v = m.v.astype(np.float32).copy()
    free = m.fixed == 0
    g = np.array([0.0, -9.8, 0.0], np.float32)
    for _ in range(steps):
        xprev = x.copy()
        v[free] = v[free] + dt32 * g
        y = x.copy()
        y[free] = x[free] + dt32 * v[free]
        x = po.solve(m, x, y, float(dtsr), iters, True, rho, init_from_inertia=True,
                     mode=po.WRAPPER).astype(np.float32)
        v[free] = ((x[free] - xprev[free]) / dt32) * np.float32(0.999)
    return x


def test_cpp_surface_matches_oracle(gpu_device, tmp_path):
    m = meshgen.beam()
    s = meshgen.BEAM_SETTINGS
    out = run_cpp(m, s["iterations"], 10, s["dt"], s["rho"], tmp_path)
    o = po.simulate(m, 10, s["dt"], s["iterations"], s["gravity"], True, s["rho"], precision=32)
    assert rel_err(out["x1"], o["x"], m) < 1e-5
    assert np.abs(out["v1"] - o["v"]).max() < 1e-3 * np.abs(o["v"]).max()
    w = wrapper_flow_oracle(m, s["iterations"], 10, s["dt"], s["rho"])
    assert rel_err(out["x2"], w, m) < 1e-5
    # per-tet materials through VBDParams::usePerTetMaterials, changed half way
    p = per_tet_flow_oracle(m, s["iterations"], 10, s["dt"], s["rho"])
    assert rel_err(out["x3"], p, m) < 1e-5
    assert rel_err(out["x3"], o["x"], m) > 1e-4  # the materials made a difference
    assert out["ncol"] == 8
    assert out["nsurf"] == 2 * 2 * (16 * 4 + 16 * 4 + 4 * 4)
    lines = open(out["obj"]).read().splitlines()
    assert sum(1 for ln in lines if ln.startswith("v ")) == m.num_verts
    assert sum(1 for ln in lines if ln.startswith("f ")) == out["nsurf"]
    # log-J elastic energy of the final state (VBDsolver::computeTotalEnergy)
    mass, trv, dm, v0 = po.mesh_setup(m.rest, m.tets, m.density, precision=64)
    X = out["x1"].astype(np.float64)
    D = np.stack([X[m.tets[:, k]] - X[m.tets[:, 0]] for k in (1, 2, 3)], axis=2)
    F = np.einsum("tij,tjk->tik", D, dm)
    J = np.abs(np.linalg.det(F))
    mu, lam = float(m.mu[0]), float(m.lam[0])
    e = np.sum(v0 * (0.5 * mu * (np.einsum("tij,tij->t", F, F) - 3) - mu * np.log(J) + 0.5 * lam * np.log(J) ** 2))
    assert abs(out["energy"] - e) <= 1e-4 * abs(e)


def _ref_cases():
    """The cases of the reference fixtures (tests/golden/make_ref_golden.py's table)."""
    spec = importlib.util.spec_from_file_location("make_ref_golden", os.path.join(GOLDEN, "make_ref_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.CASES


def run_simulate(m, iters, frames, substeps, accel, dt, rho, tmp_path, resident=False):
    if not os.path.exists(SIM_BIN):
        subprocess.run(["make", "-C", CPP_DIR], check=True, capture_output=True)
    inp = tmp_path / "sim_in.bin"
    with open(inp, "wb") as f:
        np.array([m.num_verts, m.num_tets, iters, frames, substeps, int(accel)], np.int32).tofile(f)
        np.array([m.density, m.mu[0], m.lam[0], dt, rho], np.float32).tofile(f)
        for a in (m.rest, m.x, m.v):
            a.astype(np.float32).tofile(f)
        m.tets.astype(np.int32).tofile(f)
        m.fixed.astype(np.uint8).tofile(f)
    out = tmp_path / "sim_out.bin"
    r = subprocess.run([SIM_BIN, str(inp), str(out)] + (["resident"] if resident else []), capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    raw = open(out, "rb").read()
    n3 = 3 * m.num_verts
    f = np.frombuffer(raw[: 8 * n3], np.float32)
    ints = np.frombuffer(raw[8 * n3: 8 * n3 + 16], np.int32)
    hist = np.frombuffer(raw[8 * n3 + 16:], np.float32)
    assert len(hist) == ints[3]
    return dict(x=f[:n3].reshape(-1, 3), v=f[n3:].reshape(-1, 3), callbacks=int(ints[0]), in_order=bool(ints[1]),
                positions_match=bool(ints[2]), ehist=hist.astype(np.float64))


@pytest.mark.parametrize("case", ["beam", "block_accel_off_sub2", "cube6_stiff"])
def test_simulate_matches_reference_fixtures(gpu_device, case, tmp_path):
    """VBDsolver::simulate through the C++ drop-in with a per-frame callback, against the reference's
    own VBDsolver (fixtures tests/golden/ref_trajectories.npz): positions after 10 frames within 1e-5
    of the diagonal, and energyHistory -- computeTotalEnergy after iterations 0, 10, 20, ... of every
    sub-step, VBD.cpp:93-95 -- of the same length and within 1e-4 relative (the reference evaluates it
    in FP32 through an SVD, this library in FP64 sums)."""
    make, dt, iters, accel, rho, sub = _ref_cases()[case]
    m = make()
    frames = 10
    out = run_simulate(m, iters, frames, sub, accel, dt, rho, tmp_path)
    g = np.load(os.path.join(GOLDEN, "ref_trajectories.npz"))
    assert out["callbacks"] == frames and out["in_order"] and out["positions_match"]
    err = rel_err(out["x"], g[f"{case}/x_s10"], m)
    eh = g[f"{case}/ehist"]
    print(f"simulate {case}: |x - reference|/diag {err:.3e}; energyHistory {len(out['ehist'])} values, max rel "
          f"{np.max(np.abs(out['ehist'] - eh) / np.abs(eh).max()):.2e}")
    assert err < 1e-5
    assert len(out["ehist"]) == len(eh) == frames * sub * ((iters + 9) // 10)
    np.testing.assert_allclose(out["ehist"], eh, rtol=1e-4, atol=1e-4 * np.abs(eh).max())


@pytest.mark.parametrize("case", ["beam", "block_accel_off_sub2", "cube6_stiff"])
def test_simulate_device_resident_equals_default(gpu_device, case, tmp_path):
    """VBDParams::deviceResident keeps the state on the GPU between steps (simulate reads it back
    for each callback, nothing is uploaded after the first step): the same positions, velocities and
    energyHistory bit for bit as the reference-style round trip every step."""
    make, dt, iters, accel, rho, sub = _ref_cases()[case]
    m = make()
    a = run_simulate(m, iters, 10, sub, accel, dt, rho, tmp_path)
    b = run_simulate(m, iters, 10, sub, accel, dt, rho, tmp_path, resident=True)
    assert b["callbacks"] == 10 and b["in_order"] and b["positions_match"]
    np.testing.assert_array_equal(a["x"], b["x"])
    np.testing.assert_array_equal(a["v"], b["v"])
    np.testing.assert_array_equal(a["ehist"], b["ehist"])
