"""The solver handle's API on the GPU: solveVBD / solveIteration semantics, state transfer, energies,
status counters, options and host-made fault cases (none of which faults the GPU)."""
import numpy as np
import pytest

from helpers import gpu_simulate, rel_err, small_block
from oracle import pyoracle as po
from vbd_tetmesh_b200 import GPUSolver, VBDError, build_solver, color_vertices, mesh_mass, meshgen, precompute_tets
from vbd_tetmesh_b200 import _capi

pytestmark = pytest.mark.gpu


def predicted_inertia(m, dt, g=(0.0, -9.8, 0.0)):
    """y = x + dt (v + dt g) on free vertices, y = x on pinned ones (VBDsolver::forwardStep)."""
    free = m.fixed == 0
    v = m.v.astype(np.float32).copy()
    v[free] += np.float32(dt) * np.asarray(g, np.float32)
    y = m.x.astype(np.float32).copy()
    y[free] = m.x[free] + np.float32(dt) * v[free]
    return y


@pytest.mark.parametrize("init", [_capi.INIT_FROM_POSITIONS, _capi.INIT_FROM_INERTIA])
@pytest.mark.parametrize("accel", [True, False])
def test_solve_vbd_matches_oracle(gpu_device, init, accel):
    m = small_block(seed=31)
    dt = 1 / 60
    y = predicted_inertia(m, dt)
    dtsr = np.float32(1.0 / np.float64(np.float32(dt) * np.float32(dt)))
    s = build_solver(m)
    s.update_inertia_from_cpu(y)
    s.solve_vbd(12, dtsr, accel, 0.9, init)
    x = s.get_positions()
    o = po.solve(m, m.x, y, dtsr, 12, accel, 0.9, init_from_inertia=(init == _capi.INIT_FROM_INERTIA))
    assert rel_err(x, o, m) < 1e-5
    s.close()


def test_solve_iteration_is_one_plain_sweep(gpu_device):
    m = small_block(seed=32)
    y = predicted_inertia(m, 1 / 60)
    dtsr = 3600.0
    s = build_solver(m)
    s.update_inertia_from_cpu(y)
    for _ in range(3):
        s.solve_iteration(dtsr)
    o = po.solve(m, m.x, y, dtsr, 3, False, 0.0)
    assert rel_err(s.get_positions(), o, m) < 1e-5


def test_state_round_trip(gpu_device):
    m = small_block(seed=33)
    s = build_solver(m)
    rng = np.random.default_rng(0)
    for setter, getter in ((s.set_positions, s.get_positions), (s.set_velocities, s.get_velocities),
                           (s.update_inertia_from_cpu, s.get_inertia)):
        a = rng.normal(size=(m.num_verts, 3)).astype(np.float32)
        setter(a)
        np.testing.assert_array_equal(getter(), a)


def test_device_pointer_transfer(gpu_device):
    import torch

    m = small_block(seed=34)
    s = build_solver(m)
    t = torch.randn(m.num_verts, 3, device="cuda", dtype=torch.float32)
    s.set_positions(t.data_ptr())
    out = torch.empty_like(t)
    s.get_positions(out.data_ptr())
    torch.cuda.synchronize()
    assert torch.equal(out, t)


def test_energies_match_oracle(gpu_device):
    m = small_block(seed=35, per_tet_sigma=0.2)
    dt = 1 / 60
    s = build_solver(m)
    s.step(dt, 5, (0, -9.8, 0), True, 0.9)
    x = s.get_positions().astype(np.float64)
    y = s.get_inertia().astype(np.float64)
    mass, _ = mesh_mass(m.rest, m.tets, m.density)
    dm, v0 = precompute_tets(m.rest, m.tets)
    h = float(np.float32(dt))  # the C ABI takes h as float
    ip_o = po.ip_energy(x, y, mass, m.tets, dm, v0, m.mu, m.lam, h)
    ip_g = s.energy(_capi.ENERGY_IP, h)
    assert abs(ip_g - ip_o) <= 1e-9 * abs(ip_o)
    # log-J elastic energy (VBDsolver::computeTotalEnergy)
    r = po.simulate(m, 1, dt, 5, use_acceleration=True, rho=0.9, energy_history=True)
    assert np.isfinite(s.energy(_capi.ENERGY_ELASTIC_LOGJ))
    res_g = s.energy(_capi.ENERGY_RESIDUAL, dt)
    res_o = po.residual(m, x, y, 1.0 / (dt * dt))
    assert abs(res_g - res_o) <= 1e-3 * res_o + 1e-6
    assert r["ehist"] is not None


def test_residual_decreases_with_iterations(gpu_device):
    m = small_block(seed=36)
    dt = 1 / 60
    res = []
    for iters in (2, 10, 40):
        s = build_solver(m)
        s.step(dt, iters, (0, -9.8, 0), False, 0.0)
        res.append(s.energy(_capi.ENERGY_RESIDUAL, dt))
        s.close()
    assert res[0] > res[1] > res[2]


def test_isolated_vertex_counts_singular_skip(gpu_device):
    m = meshgen.jittered_block(2, 2, 2, seed=1)
    n = m.num_verts
    # one extra vertex that belongs to no tet: zero mass, zero H, skipped by the det guard
    m.rest = np.concatenate([m.rest, [[5.0, 5.0, 5.0]]]).astype(np.float32)
    m.x = m.rest.copy()
    m.v = np.zeros_like(m.x)
    m.fixed = np.concatenate([m.fixed, [0]]).astype(np.uint8)
    s = build_solver(m)
    s.step(1 / 60, 3, (0, -9.8, 0), False, 0.0)
    x = s.get_positions()
    sing, nonf = s.status(reset=True)
    assert sing == 3 and not nonf
    np.testing.assert_array_equal(x[n], [5.0, 5.0, 5.0])
    assert s.status() == (0, False)


def test_all_pinned_mesh_does_not_move(gpu_device):
    m = meshgen.jittered_block(2, 2, 2, seed=2)
    m.fixed[:] = 1
    s = build_solver(m)
    s.step(1 / 60, 5, (0, -9.8, 0), True, 0.9)
    np.testing.assert_array_equal(s.get_positions(), m.x)


def test_degenerate_tets_are_skipped_by_the_det_guard(gpu_device):
    m = meshgen.jittered_block(1, 1, 1, seed=0, jitter=0.0)
    # collapse vertex 7 onto vertex 0: all six Kuhn tets hold both, so every V0 is 0 and Dm^-1 is
    # infinite; H becomes NaN and the |det H| > 1e-8 guard skips every vertex (VBD.cpp:141-142)
    m.rest[7] = m.rest[0]
    m.x = m.rest.copy()
    m.fixed[:] = 0
    s = build_solver(m)
    s.step(1 / 60, 2, (0, -9.8, 0), False, 0.0)
    sing, nonf = s.status()
    assert sing == 2 * m.num_verts and not nonf
    np.testing.assert_array_equal(s.get_positions(), m.x)


def test_nan_state_is_reported_nonfinite(gpu_device):
    m = small_block(seed=41)
    s = build_solver(m)
    v = np.zeros((m.num_verts, 3), np.float32)
    v[int(np.flatnonzero(m.fixed == 0)[0]), 0] = np.nan
    s.set_velocities(v)
    s.step(1 / 60, 2, (0, -9.8, 0), False, 0.0)
    _, nonf = s.status()
    assert nonf


def test_bad_colour_groups_rejected(gpu_device):
    m = small_block(seed=37)
    mass, _ = mesh_mass(m.rest, m.tets, m.density)
    dm, v0 = precompute_tets(m.rest, m.tets)
    s = GPUSolver()
    offs = np.array([0, m.num_verts], np.int32)
    verts = np.arange(m.num_verts, dtype=np.int32)
    with pytest.raises(VBDError) as e:
        s.init_from_cpu(m.x, mass, m.fixed, m.tets, offs, verts, dm, v0, m.mu, m.lam)
    assert e.value.code == 1 and "independent" in e.value.message
    _, offs, verts = color_vertices(m.num_verts, m.tets)
    verts2 = verts.copy()
    verts2[0] = verts2[1]
    with pytest.raises(VBDError) as e:
        s.init_from_cpu(m.x, mass, m.fixed, m.tets, offs, verts2, dm, v0, m.mu, m.lam)
    assert "two colour groups" in e.value.message
    with pytest.raises(VBDError) as e:
        s.step(1 / 60, 1)
    assert e.value.code == 3


def test_out_of_range_tet_rejected_before_upload(gpu_device):
    m = small_block(seed=38)
    mass, _ = mesh_mass(m.rest, m.tets, m.density)
    dm, v0 = precompute_tets(m.rest, m.tets)
    _, offs, verts = color_vertices(m.num_verts, m.tets)
    bad = m.tets.copy()
    bad[3, 2] = m.num_verts + 10
    s = GPUSolver()
    with pytest.raises(VBDError) as e:
        s.init_from_cpu(m.x, mass, m.fixed, bad, offs, verts, dm, v0, m.mu, m.lam)
    assert "outside" in e.value.message


def test_materials_required_and_updates_take_effect(gpu_device):
    m = small_block(seed=39, per_tet_sigma=0.0)
    mass, _ = mesh_mass(m.rest, m.tets, m.density)
    dm, v0 = precompute_tets(m.rest, m.tets)
    _, offs, verts = color_vertices(m.num_verts, m.tets)
    s = GPUSolver()
    s.init_from_cpu(m.x, mass, m.fixed, m.tets, offs, verts, dm, v0)
    with pytest.raises(VBDError) as e:
        s.step(1 / 60, 1)
    assert e.value.code == 3
    s.set_uniform_material(float(m.mu[0]), float(m.lam[0]))
    s.step(1 / 60, 8, (0, -9.8, 0), True, 0.9)
    soft = s.get_positions()
    o = po.simulate(m, 1, 1 / 60, 8, (0, -9.8, 0), True, 0.9)
    assert rel_err(soft, o["x"], m) < 1e-5
    # re-init replaces the mesh; stiffer per-tet material sags less
    s.init_from_cpu(m.x, mass, m.fixed, m.tets, offs, verts, dm, v0, m.mu * 10, m.lam * 10)
    s.step(1 / 60, 8, (0, -9.8, 0), True, 0.9)
    stiff = s.get_positions()
    assert stiff[:, 1].min() > soft[:, 1].min()


def test_launch_count_reported(gpu_device):
    m = small_block(seed=40)
    s = build_solver(m)
    before = s.kernel_launches()
    s.step(1 / 60, 4, (0, -9.8, 0), True, 0.9)
    s.sync()
    colour_of, _, _ = color_vertices(m.num_verts, m.tets)
    swept = len(np.unique(colour_of[m.fixed == 0]))
    assert s.kernel_launches() - before == 4 * swept + 2


def test_barrier_timeout_is_reported_not_hung(gpu_device):
    """A grid barrier that can never complete gives up after its poll limit (no hang, no fault)."""
    m = small_block(seed=42)
    s = build_solver(m)
    import ctypes as C

    out = C.c_int32(0)
    _capi.call("vbd_solver_barrier_selftest", s._h, 2000, C.byref(out))
    assert out.value == 1
    # the context stays usable
    s.set_option(_capi.OPT_PERSISTENT, 1)
    s.step(1 / 60, 4, (0, -9.8, 0), True, 0.9)
    s.sync()
    x = s.get_positions()
    assert np.all(np.isfinite(x))


def test_autotune_restores_state_and_keeps_parity(gpu_device):
    m = meshgen.cube(12)
    s = build_solver(m)
    x0 = s.get_positions()
    v0 = s.get_velocities()
    chosen = s.autotune(1 / 120, iterations=5, repeats=1)
    assert chosen["lanes"] in (2, 4, 8, 16) and chosen["layout"] in (0, 1, 2, 3, 4)
    assert chosen["persistent"] in (0, 1, 2) and chosen["record_cache"] in (0, 1)
    assert len(chosen["colour_lanes"]) == len(s.colour_groups[0]) - 1
    assert all(L in (1, 2, 4, 8, 16, 32) for L in chosen["colour_lanes"])
    np.testing.assert_array_equal(s.get_positions(), x0)
    np.testing.assert_array_equal(s.get_velocities(), v0)
    assert s.status() == (0, False)
    st = meshgen.CUBE_SETTINGS
    s.step(st["dt"], 10, st["gravity"], True, st["rho"])
    o = po.simulate(m, 1, st["dt"], 10, st["gravity"], True, st["rho"], precision=32, mode=po.CLOSED)
    assert rel_err(s.get_positions(), o["x"], m) < 1e-5


def _step_ms(s, steps, dt, iters):
    import torch

    s.step(dt, iters, (0.0, 0.0, 0.0), True, 0.9)
    s.sync()
    t = []
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        s.step(dt, iters, (0.0, 0.0, 0.0), True, 0.9)
        s.sync()
        e1.record()
        e1.synchronize()
        t.append(e0.elapsed_time(e1))
    return float(np.median(t))


def test_autotune_chooses_between_graph_and_persistent_by_time(gpu_device):
    """The autotuner's last phase times the whole step as one persistent colour-walking launch and,
    where the mesh fits, as one cluster walk, against the captured graph of separate launches, and
    keeps the fastest: re-timed afterwards, the path it kept is not slower than the others beyond
    timing noise, and every path gives the same bits at the kept lane count."""
    m = meshgen.cube(14)  # 3,375 vertices: the cluster walk fits
    s = build_solver(m)
    chosen = s.autotune(1 / 120, iterations=10, repeats=3)
    kept = chosen["persistent"]
    x0, v0 = s.get_positions(), s.get_velocities()
    t_kept = _step_ms(s, 5, 1 / 120, 10)
    x_kept = s.get_positions()
    times = {}
    for other in (0, 1, 2):
        if other == kept:
            continue
        s.set_positions(x0)
        s.set_velocities(v0)
        s.set_option(_capi.OPT_PERSISTENT, other)
        s.set_colour_lanes(None)
        times[other] = _step_ms(s, 5, 1 / 120, 10)
        # the persistent forms run VBD_OPT_LANES (at least 4) for every colour
        if chosen["lanes"] >= 4 and (kept != 0 or len(set(chosen["colour_lanes"])) == 1):
            np.testing.assert_array_equal(s.get_positions(), x_kept)
    print(f"autotune kept persistent={kept}: {t_kept:.3f} ms/step; the others {times}; {chosen}")
    assert all(t_kept <= 1.25 * t for t in times.values())
    s.close()
    assert np.all(np.isfinite(x_kept))


@pytest.mark.parametrize("lanes", [[4, 8, 16, 8, 4, 16, 8, 2], [16] * 8])
def test_per_colour_lanes_match_oracle(gpu_device, lanes):
    """Per-colour threads per vertex (vbd_solver_set_colour_lanes): within the parity bar of the
    oracle; a uniform per-colour setting equals the uniform option bit for bit."""
    m = meshgen.cube(10)
    st = meshgen.CUBE_SETTINGS
    s = build_solver(m)
    nc = len(s.get_colour_lanes())
    cl = (lanes * nc)[:nc]
    s.set_colour_lanes(cl)
    assert s.get_colour_lanes().tolist() == cl
    for _ in range(3):
        s.step(st["dt"], st["iterations"], st["gravity"], True, st["rho"])
    x = s.get_positions()
    s.close()
    o = po.simulate(m, 3, st["dt"], st["iterations"], st["gravity"], True, st["rho"], precision=32, mode=po.CLOSED)
    assert rel_err(x, o["x"], m) < 1e-5
    if len(set(cl)) == 1:
        u = gpu_simulate(m, 3, st["dt"], st["iterations"], st["gravity"], True, st["rho"], lanes=cl[0])
        np.testing.assert_array_equal(x, u["x"])


def test_colour_lanes_validation(gpu_device):
    m = small_block(seed=3)
    s = build_solver(m)
    nc = len(s.get_colour_lanes())
    with pytest.raises(VBDError):
        s.set_colour_lanes([8] * (nc + 1))
    with pytest.raises(VBDError):
        s.set_colour_lanes([3] * nc)
    s.set_colour_lanes([4] * nc)
    s.set_colour_lanes(None)
    assert s.get_colour_lanes().tolist() == [s.get_option(_capi.OPT_LANES)] * nc
    s.close()


@pytest.mark.parametrize("layout", [3, 4])
def test_record_cache_and_two_deep_prefetch_change_no_bits(gpu_device, layout):
    """The L2 policy of the record loads (evict-first, with an evict-last prefix) and the two-deep
    prefetch held to 56 registers change no arithmetic: bit-identical positions."""
    m = meshgen.cube(12)
    st = meshgen.CUBE_SETTINGS
    base = gpu_simulate(m, 2, st["dt"], st["iterations"], st["gravity"], True, st["rho"], layout=layout)
    for opts in ({_capi.OPT_RECORD_CACHE: 1}, {_capi.OPT_RECORD_CACHE: 1, _capi.OPT_RECORD_PERSIST_MB: 1},
                 {_capi.OPT_PREFETCH: 3}, {_capi.OPT_PREFETCH: 3, _capi.OPT_RECORD_CACHE: 1}):
        g = gpu_simulate(m, 2, st["dt"], st["iterations"], st["gravity"], True, st["rho"], layout=layout,
                         options=opts)
        np.testing.assert_array_equal(g["x"], base["x"])
        np.testing.assert_array_equal(g["v"], base["v"])


def test_energy_history_matches_oracle(gpu_device):
    """VBD_OPT_ENERGY_EVERY 10: vbd_solver_step appends computeTotalEnergy after iterations 0, 10, 20,
    ... of every sub-step (VBD.cpp:93-95); equal to the oracle's history within 1e-4 relative, the
    positions unchanged by it."""
    m = small_block(seed=13, dims=(7, 4, 4), per_tet_sigma=0.0)
    dt, iters, substeps, steps = 1 / 60, 25, 2, 3
    s = build_solver(m)
    s.set_option(_capi.OPT_ENERGY_EVERY, 10)
    for _ in range(steps):
        s.step(dt, iters, (0.0, -9.8, 0.0), True, 0.9, substeps)
    eh = s.energy_history(reset=False)
    assert len(eh) == steps * substeps * 3
    again = s.energy_history(reset=True)
    np.testing.assert_array_equal(eh, again)
    assert len(s.energy_history()) == 0
    x = s.get_positions()
    s.close()
    o = po.simulate(m, steps, dt, iters, (0.0, -9.8, 0.0), True, 0.9, substeps=substeps, precision=32,
                    energy_history=True)
    np.testing.assert_allclose(eh, o["ehist"][: len(eh)], rtol=1e-4, atol=1e-4 * np.abs(o["ehist"]).max())
    plain = gpu_simulate(m, steps, dt, iters, (0.0, -9.8, 0.0), True, 0.9, substeps=substeps)
    np.testing.assert_array_equal(x, plain["x"])


def test_layout_switches_rebuild_captured_graphs(gpu_device):
    """Switching the record layout frees / reallocates the streamed copy; steps replayed afterwards
    (same step parameters, so the same graph key) must use the new buffers."""
    m = small_block(seed=43)
    s = build_solver(m, layout=1)
    seq = (1, 0, 4, 3, 4, 2, 1)
    for layout in seq:
        s.set_option(_capi.OPT_LAYOUT, layout)
        s.step(1 / 60, 6, (0, -9.8, 0), True, 0.9)
    o = po.simulate(m, len(seq), 1 / 60, 6, (0, -9.8, 0), True, 0.9)
    assert rel_err(s.get_positions(), o["x"], m) < 1e-5


def test_lane_count_chosen_at_init(gpu_device):
    """Until VBD_OPT_LANES is set, init picks the lane count from the mesh: 8 for the 64^3 cube (mean
    valence 22.9, colours large enough to fill the GPU), 16 for a small mesh that leaves SMs idle,
    and an explicit setting sticks.  The record prefetch follows: the deep one (2) when no lane holds
    more than three records, else 1, unless VBD_OPT_PREFETCH is set."""
    from vbd_tetmesh_b200 import _capi

    cube = build_solver(meshgen.cube(64))
    assert cube.get_option(_capi.OPT_LANES) == 8
    # at most 24 incident tets over 8 lanes: every lane's records fit the deep prefetch
    assert cube.get_option(_capi.OPT_PREFETCH) == 2
    cube.close()
    four = build_solver(meshgen.cube(6), lanes=4)
    assert four.get_option(_capi.OPT_PREFETCH) == 1
    four.set_option(_capi.OPT_PREFETCH, 2)
    assert four.get_option(_capi.OPT_PREFETCH) == 2
    four.close()
    small = build_solver(meshgen.beam())
    assert small.get_option(_capi.OPT_LANES) == 16
    small.close()
    fixed = build_solver(meshgen.beam(), lanes=4)
    assert fixed.get_option(_capi.OPT_LANES) == 4
    fixed.close()


def _disjoint_tets(num_tets):
    """num_tets separate unit-corner tets (4 vertices each), all placed at the origin."""
    from vbd_tetmesh_b200.meshgen import Mesh

    corner = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32) * 0.05
    rest = np.tile(corner, (num_tets, 1))
    tets = np.arange(4 * num_tets, dtype=np.int32).reshape(-1, 4)
    mu, lam = meshgen.lame(1e5, 0.3)
    return Mesh(rest=rest, x=rest.copy(), v=np.zeros_like(rest), tets=tets,
                fixed=np.zeros(rest.shape[0], np.uint8), mu=np.full(num_tets, mu, np.float32),
                lam=np.full(num_tets, lam, np.float32))


def test_record_layout_chosen_at_init(gpu_device):
    """Until VBD_OPT_LAYOUT is set, init picks the 40-byte packed factored records (layout 4) when
    every vertex id fits their 21-bit fields, else the 48-byte factored records (layout 3); layout 4
    is refused for a mesh with more than 2^21 vertices, at init and afterwards."""
    small = build_solver(meshgen.cube(6))
    assert small.get_option(_capi.OPT_LAYOUT) == 4
    small.close()
    big = _disjoint_tets((1 << 19) + 1)  # 2^21 + 4 vertices
    s = build_solver(big)
    assert s.get_option(_capi.OPT_LAYOUT) == 3
    with pytest.raises(VBDError):
        s.set_option(_capi.OPT_LAYOUT, 4)
    assert s.get_option(_capi.OPT_LAYOUT) == 3
    s.step(1 / 60, 3, (0.0, -9.8, 0.0), True, 0.9)
    x = s.get_positions()
    assert np.all(np.isfinite(x)) and s.status() == (0, False)
    s.close()
    with pytest.raises(VBDError):
        build_solver(big, layout=4)
