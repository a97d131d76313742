"""Parity of the CUDA path (through the C ABI) with the oracle's restatement of VBDsolver::step.

Bar (floating point): positions after 1 and 10 steps within 1e-5 of the bounding-box diagonal of
the FP32 oracle; the incremental potential within 1e-5 relative.  Each result's error against the
FP64 oracle is printed beside it."""
import os

import numpy as np
import pytest

from helpers import gpu_simulate, rel_err, small_block
from oracle import pyoracle as po
from vbd_tetmesh_b200 import _capi, meshgen

pytestmark = pytest.mark.gpu

POS_TOL = 1e-5  # of the bounding-box diagonal
IP_TOL = 1e-5   # relative
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("steps", [1, 10])
def test_beam_matches_oracle(gpu_device, steps):
    m = meshgen.beam()
    s = meshgen.BEAM_SETTINGS
    g = gpu_simulate(m, steps, s["dt"], s["iterations"], s["gravity"], True, s["rho"])
    o32 = po.simulate(m, steps, s["dt"], s["iterations"], s["gravity"], True, s["rho"], precision=32)
    o64 = po.simulate(m, steps, s["dt"], s["iterations"], s["gravity"], True, s["rho"], precision=64)
    e32, e64 = rel_err(g["x"], o32["x"], m), rel_err(g["x"], o64["x"], m)
    print(f"beam {steps} steps: |gpu - oracle32|/diag = {e32:.3e}, |gpu - oracle64|/diag = {e64:.3e}, "
          f"|oracle32 - oracle64|/diag = {rel_err(o32['x'], o64['x'], m):.3e}")
    assert e32 < POS_TOL
    assert abs(g["ip"] - o32["ip"][-1]) <= IP_TOL * abs(o32["ip"][-1])
    vscale = max(np.abs(o64["v"]).max(), 1e-6)
    assert np.abs(g["v"] - o32["v"]).max() < 1e-3 * vscale
    assert g["singular"] == 0 and not g["nonfinite"]
    # committed FP64 fixture of the same run
    gold = np.load(os.path.join(GOLDEN, "beam_oracle.npz"))
    assert rel_err(g["x"], gold[f"x_f64_s{steps}"], m) < POS_TOL


def test_beam_100_steps_stays_close(gpu_device):
    m = meshgen.beam()
    s = meshgen.BEAM_SETTINGS
    g = gpu_simulate(m, 100, s["dt"], s["iterations"], s["gravity"], True, s["rho"])
    o = po.simulate(m, 100, s["dt"], s["iterations"], s["gravity"], True, s["rho"], precision=64, mode=po.CLOSED)
    err = rel_err(g["x"], o["x"], m)
    print(f"beam 100 steps: |gpu - oracle64|/diag = {err:.3e}")
    assert err < 1e-4


@pytest.mark.parametrize("lanes", [1, 2, 4, 8, 16, 32])
@pytest.mark.parametrize("layout", [0, 1, 2, 3, 4])
def test_launch_shapes_agree(gpu_device, lanes, layout):
    m = small_block(seed=lanes + layout)
    g = gpu_simulate(m, 3, 1 / 60, 15, (0.0, -9.8, 0.0), True, 0.9, lanes=lanes, layout=layout)
    o = po.simulate(m, 3, 1 / 60, 15, (0.0, -9.8, 0.0), True, 0.9, precision=32)
    assert rel_err(g["x"], o["x"], m) < POS_TOL


@pytest.mark.parametrize("prefetch,pdl,block", [(0, 0, 256), (1, 0, 128), (0, 1, 64), (1, 1, 128), (1, 1, 256)])
def test_prefetch_pdl_block_variants(gpu_device, prefetch, pdl, block):
    m = small_block(seed=prefetch + 2 * pdl + block)
    opts = {_capi.OPT_PREFETCH: prefetch, _capi.OPT_PDL: pdl, _capi.OPT_BLOCK: block}
    g = gpu_simulate(m, 3, 1 / 60, 15, (0.0, -9.8, 0.0), True, 0.9, options=opts)
    o = po.simulate(m, 3, 1 / 60, 15, (0.0, -9.8, 0.0), True, 0.9, precision=32)
    assert rel_err(g["x"], o["x"], m) < POS_TOL
    # prefetch, PDL and block size change no arithmetic: bit-identical to the defaults
    d = gpu_simulate(m, 3, 1 / 60, 15, (0.0, -9.8, 0.0), True, 0.9)
    np.testing.assert_array_equal(g["x"], d["x"])


@pytest.mark.parametrize("lanes,layout", [(4, 0), (8, 1), (16, 1), (32, 0), (8, 2), (4, 2), (8, 3), (16, 3), (8, 4), (4, 4)])
@pytest.mark.parametrize("accel,substeps", [(True, 1), (False, 2)])
def test_persistent_kernel_bit_identical(gpu_device, lanes, layout, accel, substeps):
    m = small_block(seed=lanes + layout, dims=(9, 5, 4), per_tet_sigma=0.2)
    kw = dict(lanes=lanes, layout=layout, options={_capi.OPT_PREFETCH: 1})
    a = gpu_simulate(m, 4, 1 / 60, 12, (0.0, -9.8, 0.0), accel, 0.9, substeps=substeps, **kw)
    kw["options"] = {_capi.OPT_PREFETCH: 1, _capi.OPT_PERSISTENT: 1}
    b = gpu_simulate(m, 4, 1 / 60, 12, (0.0, -9.8, 0.0), accel, 0.9, substeps=substeps, **kw)
    np.testing.assert_array_equal(a["x"], b["x"])
    np.testing.assert_array_equal(a["v"], b["v"])
    assert b["launches"] == 4 * substeps  # one cooperative launch per sub-step


@pytest.mark.parametrize("layout", [1, 2, 3, 4])
def test_persistent_cube_matches_graph_path(gpu_device, layout):
    m = meshgen.cube(24)
    s = meshgen.CUBE_SETTINGS
    a = gpu_simulate(m, 3, s["dt"], s["iterations"], s["gravity"], True, s["rho"], lanes=8, layout=layout)
    b = gpu_simulate(m, 3, s["dt"], s["iterations"], s["gravity"], True, s["rho"], lanes=8, layout=layout,
                     options={_capi.OPT_PERSISTENT: 1})
    np.testing.assert_array_equal(a["x"], b["x"])


@pytest.mark.parametrize("layout", [0, 1, 2, 3, 4])
def test_layouts_on_reference_fixtures(gpu_device, layout):
    """GPU vs the reference's own code (fixtures from its sources, tests/golden/make_ref_golden.py)."""
    g = np.load(os.path.join(GOLDEN, "ref_trajectories.npz"))
    m = meshgen.cube(6, seed=5)
    st = meshgen.CUBE_SETTINGS
    for steps in (1, 10):
        r = gpu_simulate(m, steps, 1 / 120, 50, (0.0, -9.8, 0.0), True, 0.9, layout=layout)
        err = rel_err(r["x"], g[f"cube6_stiff/x_s{steps}"], m)
        print(f"cube6 layout {layout} {steps} steps vs reference: {err:.3e}")
        assert err < POS_TOL


@pytest.mark.parametrize("graph", [0, 1])
def test_graph_and_direct_launches_identical(gpu_device, graph):
    m = small_block(seed=11)
    a = gpu_simulate(m, 4, 1 / 60, 10, (0.0, -9.8, 0.0), True, 0.9, graph=graph)
    b = gpu_simulate(m, 4, 1 / 60, 10, (0.0, -9.8, 0.0), True, 0.9, graph=1 - graph)
    np.testing.assert_array_equal(a["x"], b["x"])
    np.testing.assert_array_equal(a["v"], b["v"])


@pytest.mark.parametrize("accel,substeps", [(False, 1), (True, 2), (False, 3)])
def test_per_tet_materials_substeps_acceleration(gpu_device, accel, substeps):
    m = small_block(seed=21, dims=(8, 3, 3), per_tet_sigma=0.3, pin="y0")
    g = gpu_simulate(m, 10, 1 / 60, 12, (0.0, -9.8, 0.0), accel, 0.85, substeps=substeps)
    o = po.simulate(m, 10, 1 / 60, 12, (0.0, -9.8, 0.0), accel, 0.85, substeps=substeps, precision=32)
    o64 = po.simulate(m, 10, 1 / 60, 12, (0.0, -9.8, 0.0), accel, 0.85, substeps=substeps, precision=64)
    print(f"block accel={accel} substeps={substeps}: vs32 {rel_err(g['x'], o['x'], m):.3e} "
          f"vs64 {rel_err(g['x'], o64['x'], m):.3e}")
    assert rel_err(g["x"], o["x"], m) < POS_TOL


# On the stiff cube (E = 1e6, nu = 0.4, h = 1/120) the incremental potential after 10 steps is at
# the FP32 noise floor: over seeds 1-8 the FP32 oracle (bit-exact to the reference's build) itself
# lies 2e-6 .. 4.6e-5 from the FP64 run, and FP32 GPU results of every record layout and lane count
# scatter by the same amount.  Positions stay within 3.3e-7 of the bounding-box diagonal.  So the
# energy here is checked against FP64 within that envelope; the 1e-5 energy bar against the FP32
# oracle applies to the beam configurations above.
STIFF_IP_TOL_F64 = 6e-5


@pytest.mark.parametrize("seed", range(1, 9))
def test_initial_velocity_and_stiff_material(gpu_device, seed):
    m = meshgen.cube(6, E=1e6, nu=0.4, seed=seed)
    s = meshgen.CUBE_SETTINGS
    g = gpu_simulate(m, 10, s["dt"], s["iterations"], s["gravity"], True, s["rho"])
    o = po.simulate(m, 10, s["dt"], s["iterations"], s["gravity"], True, s["rho"], precision=32, mode=po.CLOSED)
    o64 = po.simulate(m, 10, s["dt"], s["iterations"], s["gravity"], True, s["rho"], precision=64, mode=po.CLOSED)
    ip32, ip64 = o["ip"][-1], o64["ip"][-1]
    print(f"cube6 seed {seed} 10 steps: x vs32 {rel_err(g['x'], o['x'], m):.3e} vs64 {rel_err(g['x'], o64['x'], m):.3e}; "
          f"IP vs32 {abs(g['ip'] - ip32) / abs(ip32):.2e} vs64 {abs(g['ip'] - ip64) / abs(ip64):.2e} "
          f"(oracle32 vs64 {abs(ip32 - ip64) / abs(ip64):.2e})")
    assert rel_err(g["x"], o["x"], m) < POS_TOL
    assert abs(g["ip"] - ip64) <= STIFF_IP_TOL_F64 * abs(ip64)
    assert abs(ip32 - ip64) <= STIFF_IP_TOL_F64 * abs(ip64)


@pytest.mark.parametrize("layout,lanes", [(3, 8), (4, 8), (4, 4), (4, 16)])
def test_deep_prefetch_bit_identical(gpu_device, layout, lanes):
    """VBD_OPT_PREFETCH 2 loads a lane's first three records before the dependency wait and any
    further ones where they are used (4 lanes hold up to six on the cube); the summation order is
    unchanged, so positions equal those of prefetch 0 and 1 bit for bit."""
    m = meshgen.cube(12)
    s = meshgen.CUBE_SETTINGS
    out = [gpu_simulate(m, 2, s["dt"], s["iterations"], s["gravity"], True, s["rho"], layout=layout, lanes=lanes,
                        options={_capi.OPT_PREFETCH: pf})["x"] for pf in (2, 1, 0)]
    np.testing.assert_array_equal(out[0], out[1])
    np.testing.assert_array_equal(out[0], out[2])


def test_l2_prefetch_option_changes_no_result(gpu_device):
    """VBD_OPT_L2_PREFETCH only warms L2 with the next colour's records: bit-identical results."""
    m = meshgen.cube(12)
    s = meshgen.CUBE_SETTINGS
    out = []
    for pf in (0, 1):
        for layout in (2, 3, 4):
            g = gpu_simulate(m, 2, s["dt"], s["iterations"], s["gravity"], True, s["rho"], layout=layout,
                             options={_capi.OPT_L2_PREFETCH: pf})
            out.append(g["x"])
    for k in range(3):
        np.testing.assert_array_equal(out[k], out[k + 3])
