"""The cluster-resident colour walk (VBD_OPT_PERSISTENT 2): one thread-block cluster per sub-step,
the mesh's positions in distributed shared memory, colours handed over by st.async stores that
complete on the receiving CTA's mbarrier.  Its arithmetic and lane-to-record assignment are the
captured graph's, so positions, velocities and adjoint gradients must equal the graph path's bit
for bit at the same lane count and layout, for any number of CTAs (which changes only which group
sweeps which vertex); meshes that do not fit are refused on the host."""
import numpy as np
import pytest

from helpers import gpu_simulate, rel_err, small_block
from oracle import pyoracle as po
from vbd_tetmesh_b200 import _capi, build_solver, meshgen

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("lanes", [4, 8, 16, 32])
@pytest.mark.parametrize("layout", [3, 4])
@pytest.mark.parametrize("accel,substeps", [(True, 1), (False, 2)])
def test_cluster_walk_bit_identical_to_graph(gpu_device, lanes, layout, accel, substeps):
    m = small_block(seed=lanes + layout, dims=(9, 5, 4), per_tet_sigma=0.2)
    kw = dict(lanes=lanes, layout=layout, options={_capi.OPT_PREFETCH: 1})
    a = gpu_simulate(m, 4, 1 / 60, 12, (0.0, -9.8, 0.0), accel, 0.9, substeps=substeps, **kw)
    kw["options"] = {_capi.OPT_PREFETCH: 1, _capi.OPT_PERSISTENT: 2}
    b = gpu_simulate(m, 4, 1 / 60, 12, (0.0, -9.8, 0.0), accel, 0.9, substeps=substeps, **kw)
    np.testing.assert_array_equal(a["x"], b["x"])
    np.testing.assert_array_equal(a["v"], b["v"])
    assert b["launches"] == 4 * substeps  # one cluster launch per sub-step
    assert b["singular"] == 0 and not b["nonfinite"]


@pytest.mark.parametrize("ctas", [1, 2, 5, 16])
def test_cluster_ctas_change_no_bits(gpu_device, ctas):
    """With 1 CTA the differentiated beam's colours (about 330 vertices at 16 lanes) take several
    rounds per colour; with 16 one or two.  Same bits as the graph path either way."""
    m = meshgen.diff_beam()[0]
    st = meshgen.DIFF_SETTINGS
    a = gpu_simulate(m, 3, st["dt"], st["iterations"], st["gravity"], True, st["rho"], lanes=16, layout=4)
    b = gpu_simulate(m, 3, st["dt"], st["iterations"], st["gravity"], True, st["rho"], lanes=16, layout=4,
                     options={_capi.OPT_PERSISTENT: 2, _capi.OPT_CLUSTER_CTAS: ctas})
    np.testing.assert_array_equal(a["x"], b["x"])
    np.testing.assert_array_equal(a["v"], b["v"])


def test_cluster_walk_beam_matches_oracle(gpu_device):
    m = meshgen.beam()
    s = meshgen.BEAM_SETTINGS
    g = gpu_simulate(m, 10, s["dt"], s["iterations"], s["gravity"], True, s["rho"], layout=4,
                     options={_capi.OPT_PERSISTENT: 2})
    o32 = po.simulate(m, 10, s["dt"], s["iterations"], s["gravity"], True, s["rho"], precision=32)
    o64 = po.simulate(m, 10, s["dt"], s["iterations"], s["gravity"], True, s["rho"], precision=64)
    e32, e64 = rel_err(g["x"], o32["x"], m), rel_err(g["x"], o64["x"], m)
    print(f"beam 10 steps, cluster walk: vs oracle32 {e32:.3e}, vs oracle64 {e64:.3e}")
    assert e32 < 1e-5
    assert abs(g["ip"] - o32["ip"][-1]) <= 1e-5 * abs(o32["ip"][-1])


@pytest.mark.parametrize("init_mode", [_capi.INIT_FROM_POSITIONS, _capi.INIT_FROM_INERTIA])
def test_cluster_solve_bit_identical(gpu_device, init_mode):
    m = small_block(seed=7, dims=(8, 4, 4))
    out = []
    for opts in ({}, {_capi.OPT_PERSISTENT: 2}):
        s = build_solver(m, lanes=8, layout=4)
        for k, v in opts.items():
            s.set_option(k, v)
        y = s.get_positions() + np.float32(1e-3)
        s.update_inertia_from_cpu(y)
        s.solve_vbd(25, 3600.0, True, 0.9, init_mode)
        s.sync()
        out.append(s.get_positions())
        s.close()
    np.testing.assert_array_equal(out[0], out[1])


@pytest.mark.parametrize("alternate,adj_rho", [(0, 0.9), (1, 0.0), (0, 0.0)])
@pytest.mark.parametrize("layout", [3, 4])
def test_cluster_adjoint_gradients_equal_graph(gpu_device, alternate, adj_rho, layout):
    """With the cluster walk the backward recomputes the recorded forward segments through the
    same walk and runs each sub-step's adjoint sweeps as one cluster launch; the gradients equal the
    launch-per-colour path's bit for bit."""
    m = meshgen.jittered_block(6, 3, 3, seed=3, per_tet_sigma=0.2, E=2e4)
    W = np.random.default_rng(3).normal(size=(m.num_verts, 3))
    grads = []
    for walk in (0, 2):
        s = build_solver(m, lanes=8, layout=layout)
        s.set_option(_capi.OPT_ADJOINT_ALTERNATE, alternate)
        s.set_option(_capi.OPT_PERSISTENT, walk)
        s.record(2)
        for _ in range(5):
            s.step(1 / 60, 40, (0.0, -9.8, 0.0), True, 0.9)
        l0 = s.kernel_launches()
        grads.append(s.backward(W, None, 60, adj_rho))
        launches = s.kernel_launches() - l0
        s.close()
        if walk == 2:
            # per sub-step: rhs, one adjoint walk, parameter gradients, pinned coupling, velocity
            # update; plus one walk per recomputed sub-step
            assert launches < 100  # the launch-per-colour path: over 2,400
    for a, b in zip(grads[0], grads[1]):
        np.testing.assert_array_equal(a, b)


def test_cluster_walk_diff_beam_adjoint_matches_graph(gpu_device):
    """The differentiated beam at its stated configuration (30 steps x 30 iterations, checkpoint
    10, 50 adjoint sweeps): the cluster walk's positions and gradients equal the launch-per-colour
    path's."""
    m, tip, target = meshgen.diff_beam()
    st = meshgen.DIFF_SETTINGS
    runs = []
    for walk in (0, 2):
        s = build_solver(m, lanes=8, layout=3)
        s.set_option(_capi.OPT_PERSISTENT, walk)
        s.record(st["checkpoint"])
        for _ in range(st["steps"]):
            s.step(st["dt"], st["iterations"], st["gravity"], True, st["rho"])
        x = s.get_positions().astype(np.float64)
        g = np.zeros((m.num_verts, 3))
        g[tip] = 2.0 * (x[tip] - target)
        runs.append((x, s.backward(g, None, st["adjoint_iterations"], st["adjoint_rho"])))
        s.close()
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    for a, b in zip(runs[0][1], runs[1][1]):
        np.testing.assert_array_equal(a, b)


def test_cluster_walk_refuses_meshes_that_do_not_fit(gpu_device):
    # 25^3 vertices x 48 B = 750 KB of positions: more than one CTA's shared memory
    s = build_solver(meshgen.cube(24), layout=4)
    with pytest.raises(_capi.VBDError) as e:
        s.set_option(_capi.OPT_PERSISTENT, 2)
    assert e.value.code == 1  # VBD_ERR_INVALID_ARG
    s.close()
    # the gathered tet records are not read by the cluster walk
    s = build_solver(small_block(seed=1), layout=2)
    with pytest.raises(_capi.VBDError):
        s.set_option(_capi.OPT_PERSISTENT, 2)
    s.close()
    s = build_solver(small_block(seed=1), layout=4)
    s.set_option(_capi.OPT_PERSISTENT, 2)
    s.set_option(_capi.OPT_LAYOUT, 2)
    with pytest.raises(_capi.VBDError):
        s.step(1 / 60, 5, (0.0, -9.8, 0.0), True, 0.9)
    s.close()


def test_beam_autotune_with_cluster_candidates_completes(gpu_device):
    """The autotuner on the beam tries the cluster walk with up to 9 CTAs for colours of 29-72
    vertices, so CTAs finish a colour at very different times.  Every colour's bytes must be
    announced on the receiving CTA before any CTA can send them; an earlier announcement order let
    st.async bytes arrive first, and a bounded mbarrier wait gave up (VBD_ERR_TIMEOUT)."""
    m = meshgen.beam()
    st = meshgen.BEAM_SETTINGS
    s = build_solver(m)
    for _ in range(2):
        chosen = s.autotune(st["dt"], iterations=st["iterations"], repeats=5)
        assert chosen["persistent"] in (0, 1, 2)
    s.step(st["dt"], st["iterations"], st["gravity"], True, st["rho"])
    s.sync()
    assert s.status() == (0, False)
    s.close()


def test_cluster_forward_with_launch_per_colour_adjoint(gpu_device):
    """4,096 vertices: the forward walk fits (48 B per vertex) but the adjoint walk (64 B) does not,
    so the backward recomputes through the cluster walk and sweeps the adjoint colour by colour;
    the gradients still equal the launch-per-colour path's."""
    m = meshgen.jittered_block(15, 15, 15, seed=5, per_tet_sigma=0.2, E=5e4)
    assert m.num_verts == 4096
    W = np.random.default_rng(5).normal(size=(m.num_verts, 3))
    grads = []
    for walk in (0, 2):
        s = build_solver(m, lanes=8, layout=4)
        s.set_option(_capi.OPT_PERSISTENT, walk)
        s.record(2)
        for _ in range(3):
            s.step(1 / 60, 20, (0.0, -9.8, 0.0), True, 0.9)
        grads.append(s.backward(W, None, 30, 0.9))
        s.close()
    for a, b in zip(grads[0], grads[1]):
        np.testing.assert_array_equal(a, b)


def test_cluster_walk_with_energy_history_runs_separate_launches(gpu_device):
    """A step that must append VBDsolver's energy history runs as separate launches even with the
    cluster walk selected, and its positions and energies equal the graph path's."""
    m = meshgen.beam()
    st = meshgen.BEAM_SETTINGS
    out = []
    for walk in (0, 2):
        s = build_solver(m, lanes=16, layout=3)
        s.set_option(_capi.OPT_PERSISTENT, walk)
        s.set_option(_capi.OPT_ENERGY_EVERY, 10)
        for _ in range(3):
            s.step(st["dt"], st["iterations"], st["gravity"], True, st["rho"])
        out.append((s.get_positions(), s.energy_history()))
        s.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    assert len(out[1][1]) == 3 * 2
    np.testing.assert_array_equal(out[0][1], out[1][1])


def test_cluster_walk_refuses_a_reinitialised_mesh_that_does_not_fit(gpu_device):
    from vbd_tetmesh_b200 import color_vertices, mesh_mass, precompute_tets

    s = build_solver(small_block(seed=2), layout=4)
    s.set_option(_capi.OPT_PERSISTENT, 2)
    s.step(1 / 60, 5, (0.0, -9.8, 0.0), True, 0.9)
    big = meshgen.cube(24)
    _, offs, verts = color_vertices(big.num_verts, big.tets)
    mass, _ = mesh_mass(big.rest, big.tets, big.density)
    dminv, v0 = precompute_tets(big.rest, big.tets)
    s.init_from_cpu(big.x, mass, big.fixed, big.tets, offs, verts, dminv, v0, big.mu, big.lam)
    with pytest.raises(_capi.VBDError) as e:
        s.step(1 / 120, 5, (0.0, -9.8, 0.0), True, 0.9)
    assert e.value.code == 1  # VBD_ERR_INVALID_ARG: does not fit
    s.set_option(_capi.OPT_PERSISTENT, 0)
    s.step(1 / 120, 5, (0.0, -9.8, 0.0), True, 0.9)
    s.sync()
    assert np.all(np.isfinite(s.get_positions()))
    s.close()


@pytest.mark.parametrize("case,lanes,layout,ctas", [("beam", 16, 3, 0), ("beam", 32, 4, 0), ("diff", 8, 4, 16),
                                                    ("block", 4, 3, 3), ("diff", 16, 4, 1)])
def test_resident_records_change_no_bits(gpu_device, case, lanes, layout, ctas):
    """VBD_OPT_CLUSTER_RESIDENT 1 keeps each CTA's element records, inertial targets and spans in its
    shared memory where they fit (the differentiated beam at 8 lanes only with 16 CTAs; with one
    CTA they do not fit and the walk reads them from L2); 0 always reads them from L2.  Both equal
    the captured graph bit for bit."""
    if case == "beam":
        m, st = meshgen.beam(), meshgen.BEAM_SETTINGS
    elif case == "diff":
        m, st = meshgen.diff_beam()[0], meshgen.DIFF_SETTINGS
    else:
        m, st = small_block(seed=9, dims=(9, 5, 4)), dict(dt=1 / 60, iterations=15, rho=0.9, gravity=(0.0, -9.8, 0.0))
    args = (m, 3, st["dt"], st["iterations"], st["gravity"], True, st["rho"])
    graph = gpu_simulate(*args, lanes=lanes, layout=layout)
    for resident in (1, 0):
        w = gpu_simulate(*args, lanes=lanes, layout=layout,
                         options={_capi.OPT_PERSISTENT: 2, _capi.OPT_CLUSTER_CTAS: ctas,
                                  _capi.OPT_CLUSTER_RESIDENT: resident})
        np.testing.assert_array_equal(graph["x"], w["x"])
        np.testing.assert_array_equal(graph["v"], w["v"])
        assert w["singular"] == 0 and not w["nonfinite"]
