#!/usr/bin/env python
"""Benchmark of the VBD hot path on B200: vertex-iterations/s on the 64^3 jittered cube.

Workload (one "step"): one VBDsolver::step of the 274,625-vertex / 1,572,864-tet cube -- predictor,
50 Gauss-Seidel colour sweeps with the Chebyshev blend (rho 0.9), velocity update -- dt = 1/120 s,
E = 1e6 Pa, nu = 0.4, density 1000, bottom face pinned, seeded initial velocities, gravity -9.8 y.

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

* value: whole-job vertex-iterations/s (all vertices x iterations x steps over all ranks / max over
  ranks of the device-timed region), inputs resident in HBM, L2 flushed (256 MiB write) between
  timed steps outside the timed events.
* e2e: the same metric through the C ABI with host buffers: each step uploads positions and
  velocities from pinned host memory, steps, and reads both back.
* roofline: the colour-sweep kernel (400 of a step's 402 launches): its algorithmic bytes per launch
  (60 B per incident tet + 96 B per swept vertex) over the timed region's CUDA-event time per sweep
  launch; a second pass with an event pair around every sweep launched on its own is reported
  beside it as "isolated".
* cpu_baseline (rank 0, N = 1): the reference's own CPU sources (oracle/_ref, compiled against the
  Eigen-API subset) on all host cores, one cube iteration per sample; the oracle's reference-cost
  restatement (literal 12x12 element Hessian, energy every 10 iterations) when they are not built.
* --impl reference: that CPU implementation alone (rank 0), each step one cube iteration.
* N > 1 (torchrun): one replica of the cube per GPU ("replicas only": a single mesh does not
  shard); no collective on the data path, barrier + max-over-ranks timing.
"""
from __future__ import annotations

import argparse
import json
import os
import signal
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "VBD vertex-iters/s on 1 B200 at stated tol; batched vs plain; adjoint/forward"
UNIT = "vertex-iterations/s"
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cube", type=int, default=64, help="cells per cube edge")
    ap.add_argument("--iterations", type=int, default=50)
    ap.add_argument("--lanes", type=int, default=None)
    ap.add_argument("--layout", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batch-meshes", type=int, default=512)
    ap.add_argument("--batch-steps", type=int, default=3)
    ap.add_argument("--no-autotune", action="store_true", help="time the launch configuration chosen at init")
    ap.add_argument("--colour-lanes", default=None,
                    help="comma-separated threads per vertex of each colour of the cube (with --no-autotune)")
    ap.add_argument("--record-cache", type=int, default=None, help="VBD_OPT_RECORD_CACHE of the cube solver")
    ap.add_argument("--persist-mb", type=int, default=None, help="VBD_OPT_RECORD_PERSIST_MB of the cube solver")
    ap.add_argument("--prefetch", type=int, default=None, help="VBD_OPT_PREFETCH of the cube solver")
    ap.add_argument("--no-plain", action="store_true",
                    help="batched section without the per-mesh solvers it is compared with (for profiling)")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-material-id", action="store_true")
    ap.add_argument("--clocks-dir", default=None,
                    help="directory for the raw nvidia-smi clock samples (default: a temporary directory)")
    return ap.parse_args()


def workload_config(mesh, iters):
    return {
        "workload": f"cube{mesh.dims[0]} jittered Kuhn-split grid, VBDsolver::step x steps",
        "vertices": mesh.num_verts,
        "tets": mesh.num_tets,
        "pinned": int(mesh.fixed.sum()),
        "iterations_per_step": iters,
        "dt": 1.0 / 120.0,
        "chebyshev_rho": 0.9,
        "E": 1e6,
        "nu": 0.4,
        "density": 1000.0,
        "jitter": 0.2,
        "seed": 1234,
        "gravity": [0.0, -9.8, 0.0],
        "l2": "flushed between timed steps (256 MiB write, outside the events)",
    }


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def cpu_reference(mesh, samples, warmup=0):
    """Times the reference's CPU VBD path on all host threads, one cube iteration per sample.

    Prefers the reference's own sources (oracle/_ref: TetMesh / VBDsolver compiled against the
    Eigen-API subset, numThreads = host cores, i.e. its OpenMP loop over colours, VBD.cpp:120);
    falls back to the oracle's reference-cost restatement (literal 12x12 element Hessian, OpenMP
    within each colour).  Returns (vertex-iters/s, threads, seconds, kind, sample description)."""
    from oracle import pyoracle as po

    threads = max(1, os.cpu_count() or 1)
    s = meshgen_settings()
    if po.ref_available():
        h = po.RefHandle(mesh, s["dt"], s["iterations"], s["gravity"], True, s["rho"], threads=threads)
        run = lambda: h.iterations(1)  # noqa: E731
        kind = "reference"
        what = ("the reference's own TetMesh/VBDsolver sources (compiled against the Eigen-API subset), "
                "VBDsolver::step's iteration loop one iteration per sample: colour sweep with the literal 12x12 "
                "element Hessian, Chebyshev, computeTotalEnergy every 10th iteration, predictor / velocity "
                "update every 50th; numThreads = host cores (its OpenMP loop over colours)")
    else:
        h = po.Handle(mesh, po.LITERAL_FULL12, threads)
        k = [0]

        def run():
            h.step(1, s["dt"], 1, s["gravity"], True, s["rho"], energy=(k[0] % 10 == 0))
            k[0] += 1

        kind = "port"
        what = ("the oracle's reference-cost restatement: literal 12x12 element Hessian per incidence, energy "
                "every 10th iteration, OpenMP within each colour")
    for _ in range(warmup):
        run()
    times = []
    for _ in range(samples):
        t0 = time.perf_counter()
        run()
        times.append(time.perf_counter() - t0)
    h.close()
    total = sum(times)
    return mesh.num_verts * samples / total, threads, total, kind, what


def cpu_restatement(cube_mesh):
    """The oracle's reference-cost restatement of the reference CPU path (literal 12x12 element
    Hessian per incidence, computeTotalEnergy every 10th iteration, VBD.cpp:60-203), race-free:
    OpenMP within each colour, the same results at any thread count.  Timed at 1 thread and at all
    host threads on
      * the beam (16x4x4 cells, 425 vertices), 100 steps x 20 iterations in full, and
      * the cube, one full step (50 iterations) at all threads; at 1 thread (about 8 s per
        iteration) from one iteration without and one with the energy evaluation, extrapolated to
        the step's 50 iterations and 5 energy evaluations.
    Returns the runs in vertex-iterations/s."""
    from oracle import pyoracle as po
    from vbd_tetmesh_b200 import meshgen

    allc = max(1, po.max_threads())
    runs = []
    beam, bs = meshgen.beam(), meshgen.BEAM_SETTINGS
    for thr in (1, allc):
        h = po.Handle(beam, po.LITERAL_FULL12, thr)
        t0 = time.perf_counter()
        h.step(100, bs["dt"], bs["iterations"], bs["gravity"], True, bs["rho"], energy=True)
        t = time.perf_counter() - t0
        h.close()
        runs.append({"workload": "beam 16x4x4 cells (425 vertices), 100 steps x 20 iterations, in full",
                     "threads": thr, "seconds": t, "value": beam.num_verts * 20 * 100 / t})
    cs = meshgen.CUBE_SETTINGS
    n = cube_mesh.num_verts
    h = po.Handle(cube_mesh, po.LITERAL_FULL12, 1)
    t0 = time.perf_counter()
    h.step(1, cs["dt"], 1, cs["gravity"], True, cs["rho"], energy=False)
    t_it = time.perf_counter() - t0
    t0 = time.perf_counter()
    h.step(1, cs["dt"], 1, cs["gravity"], True, cs["rho"], energy=True)
    t_en = max(time.perf_counter() - t0 - t_it, 0.0)
    h.close()
    t_step = 50 * t_it + 5 * t_en
    runs.append({"workload": "cube 64^3 (274,625 vertices), one step of 50 iterations, extrapolated from one "
                             "iteration without and one with the energy evaluation",
                 "threads": 1, "seconds": t_step, "value": n * 50 / t_step, "measured_seconds": t_it + t_it + t_en})
    h = po.Handle(cube_mesh, po.LITERAL_FULL12, allc)
    t0 = time.perf_counter()
    h.step(1, cs["dt"], 50, cs["gravity"], True, cs["rho"], energy=True)
    t = time.perf_counter() - t0
    h.close()
    runs.append({"workload": "cube 64^3 (274,625 vertices), one full step of 50 iterations", "threads": allc,
                 "seconds": t, "value": n * 50 / t})
    return {"kind": "port", "unit": UNIT, "host_threads": allc,
            "what": "the oracle's reference-cost restatement of VBDsolver::step: literal 12x12 element Hessian per "
                    "incidence, computeTotalEnergy every 10th iteration, OpenMP within each colour (race-free)",
            "runs": runs}


def meshgen_settings():
    from vbd_tetmesh_b200 import meshgen

    return meshgen.CUBE_SETTINGS


def nvsmi_device(local: int) -> str:
    """nvidia-smi's name for CUDA device `local` of this process: the local-th entry of
    CUDA_VISIBLE_DEVICES when that is set (an index or a UUID, both of which nvidia-smi --id
    takes), else the index itself."""
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    ids = [v.strip() for v in vis.split(",") if v.strip()]
    return ids[local] if local < len(ids) else str(local)


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region (device_index is the CUDA
    device of this process; the sampler reads the same GPU under any CUDA_VISIBLE_DEVICES)."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index, out_dir=None):
        self.device_index = device_index
        self.out_dir = out_dir
        self.proc = None
        self.path = None

    def start(self):
        try:
            out_dir = self.out_dir or tempfile.mkdtemp(prefix="vbd_bench_clocks_")
            os.makedirs(out_dir, exist_ok=True)
            self.path = os.path.join(out_dir, f"clocks_rank{self.device_index}.csv")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={nvsmi_device(self.device_index)}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def _lines(self):
        try:
            return open(self.path).read().splitlines()
        except Exception:
            return []

    def wait_first_sample(self, timeout=5.0):
        t0 = time.time()
        while self.proc is not None and not self._lines() and time.time() - t0 < timeout:
            time.sleep(0.05)

    def mark(self):
        """Samples from here on belong to the timed passes."""
        self.first = len(self._lines())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.send_signal(signal.SIGTERM)
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in self._lines()[getattr(self, "first", 0):]:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f[5], f[6], f[7], f[8]))
            except ValueError:
                continue
        if not rows:
            return None
        sm = sorted(r[0] for r in rows)
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            for name, val in zip(names, r[2:]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": max(r[1] for r in rows), "reasons": sorted(reasons),
                "samples": len(rows)}


def wrapper_workload(mesh):
    """One VBD_GPU_Solver::solveVBD call on the cube as main.cpp issues it: inertial target
    y = x + N(0, 1e-3 m) on free vertices (seed 7), 1/h^2 = 14400 (h = 1/120), 50 iterations,
    Chebyshev rho 0.9, starting from x = y."""
    import numpy as np

    rng = np.random.default_rng(7)
    y = (mesh.x + 1e-3 * rng.normal(size=mesh.x.shape)).astype(np.float32)
    y[mesh.fixed == 1] = mesh.x[mesh.fixed == 1]
    return y, 14400.0, 50, 0.9


def run_reference(args):
    """--impl reference: the reference's CPU implementation of the path, timed on the host (rank 0)."""
    from vbd_tetmesh_b200 import meshgen

    mesh = meshgen.cube(args.cube)
    value, cores, total, kind, what = cpu_reference(mesh, args.steps, warmup=args.warmup)
    cfg = workload_config(mesh, args.iterations)
    cfg["sample"] = "each step = one iteration (colour sweep) of the cube's 50-iteration VBDsolver::step loop"
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": cfg,
        "cpu_baseline": {
            "value": value,
            "unit": UNIT,
            "cores": cores,
            "kind": kind,
            "sample": f"{args.steps} samples of 1 cube iteration (274,625 vertices): {what}",
        },
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    gpu = reference_gpu_wrapper(mesh)
    if gpu is not None:
        line["gpu_wrapper"] = gpu
    print(json.dumps(line), flush=True)


def reference_gpu_wrapper(mesh):
    """The reference's own GPU path (VBD_GPU_Solver::solveVBD, its 16-thread-per-vertex kernels)
    on the wrapper workload, when its library was built (oracle/_ref/libvbdref_gpu.so) and a GPU is
    present; device time from CUDA events on the stream it launches on."""
    try:
        import torch

        if not torch.cuda.is_available():
            return None
        from oracle import pyoracle as po

        if not po.ref_gpu_available():
            return None
    except ImportError:
        return None
    y, dtsr, iters, rho = wrapper_workload(mesh)
    h = po.RefGpuHandle(mesh, iterations=iters, rho=rho)
    h.set_inertia(y)
    h.solve(iters, dtsr, True, rho)
    ms = sorted(h.solve(iters, dtsr, True, rho) for _ in range(5))
    h.close()
    med = ms[len(ms) // 2]
    return {
        "workload": "one VBD_GPU_Solver::solveVBD on the cube (y = x + N(0, 1e-3), 1/h^2 14400, 50 iterations, "
                    "rho 0.9, from x = y): the reference's own kernels",
        "ms_per_solve": med,
        "value": mesh.num_verts * iters / (med * 1e-3),
        "unit": UNIT,
    }


def bench_wrapper(mesh, local, stream):
    """This project's VBD_OPT_SEMANTICS = 1 path (the reference GPU wrapper's arithmetic, bit-identical
    to its kernels on this workload in tests/test_gpu_wrapper_mode.py) on the wrapper workload."""
    import torch

    from vbd_tetmesh_b200 import _capi, build_solver

    y, dtsr, iters, rho = wrapper_workload(mesh)
    out = {"workload": "one solveVBD on the cube (y = x + N(0, 1e-3), 1/h^2 14400, 50 iterations, rho 0.9, "
                       "from x = y) with the reference GPU wrapper's semantics"}
    with torch.cuda.stream(stream):
        for layout in (0, 1):
            s = build_solver(mesh, device=local, stream=stream.cuda_stream, layout=layout)
            s.set_option(_capi.OPT_SEMANTICS, 1)
            s.update_inertia_from_cpu(y)
            s.solve_vbd(iters, dtsr, True, rho, _capi.INIT_FROM_INERTIA)
            s.sync()
            ms = []
            for _ in range(5):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                s.solve_vbd(iters, dtsr, True, rho, _capi.INIT_FROM_INERTIA)
                e1.record(stream)
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
            s.close()
            med = sorted(ms)[len(ms) // 2]
            out[f"layout{layout}"] = {"ms_per_solve": med, "value": mesh.num_verts * iters / (med * 1e-3), "unit": UNIT}
    return out


def bench_batched(args, rank, world, local, stream, dist, barrier):
    """The batched configuration: args.batch_meshes jittered blocks (dims U{4..24}^3, E log-uniform
    [1e4, 1e6], nu U[0.2, 0.45], one face pinned), dt 1/60, 20 iterations, Chebyshev 0.9.  One solver
    over the concatenated meshes (colour c of every mesh in one launch) against one plain solver per
    mesh stepped mesh after mesh on the same stream.  Whole meshes are sharded across ranks,
    balanced by tet count; times are the max over ranks."""
    import torch

    from vbd_tetmesh_b200 import _capi, build_batch_solver, build_solver, meshgen
    from vbd_tetmesh_b200.sharding import combine_over_ranks, shard_meshes

    meshes = meshgen.batched_blocks(args.batch_meshes)
    sub = [meshes[k] for k in shard_meshes([m.num_tets for m in meshes], world)[rank]]
    b = meshgen.concat(sub)
    dt, iters, rho, g = 1.0 / 60.0, 20, 0.9, (0.0, -9.8, 0.0)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    K = args.batch_steps

    def timed(step_fn, label):
        step_fn()  # warm-up (graph capture)
        torch.cuda.synchronize()
        barrier()
        ms = 0.0
        torch.cuda.nvtx.range_push(label)
        for _ in range(K):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step_fn()
            e1.record(stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
        torch.cuda.nvtx.range_pop()
        barrier()
        return ms

    with torch.cuda.stream(stream):
        bs = build_batch_solver(b, device=local, stream=stream.cuda_stream)
        tuned = None if args.no_autotune else bs.autotune(dt, iterations=iters, repeats=3)
        batch_colour_lanes = bs.get_colour_lanes()
        l0 = bs.kernel_launches()
        ms_b = timed(lambda: bs.step(dt, iters, g, True, rho), "batched_timed")
        launches_b = (bs.kernel_launches() - l0) // (K + 1)
        xb = bs.get_positions()
        batch_lanes = bs.get_option(_capi.OPT_LANES)
        batch_layout = bs.get_option(_capi.OPT_LAYOUT)
        # algorithmic bytes of one step's colour sweeps (60 B per incidence + 96 B per swept vertex),
        # from a pass with an event pair around every sweep (after the positions were read)
        bs.set_option(_capi.OPT_KERNEL_TIMING, 1)
        bs.kernel_time(reset=True)
        flush.fill_(1.0)
        bs.step(dt, iters, g, True, rho)
        sw_ms, sw_launches, sw_bytes = bs.kernel_time(reset=True)
        bs.close()
        # the per-mesh solvers use the batch solver's lane count and record layout, so each mesh's
        # arithmetic (and result) is the batch's
        if args.no_plain:
            ms_p, launches_p, xp = float("nan"), 0, xb
        else:
            plain = [build_solver(m, device=local, stream=stream.cuda_stream, lanes=batch_lanes, layout=batch_layout)
                     for m in sub]
            for p in plain:  # colour c of a mesh is swept with the batch's shape for colour c
                p.set_colour_lanes(batch_colour_lanes[: len(p.get_colour_lanes())])
            l0 = sum(p.kernel_launches() for p in plain)

            def plain_step():
                for p in plain:
                    p.step(dt, iters, g, True, rho)

            ms_p = timed(plain_step, "plain_timed")
            launches_p = (sum(p.kernel_launches() for p in plain) - l0) // (K + 1)
            xp = np.concatenate([p.get_positions() for p in plain])
            for p in plain:
                p.close()
    same = bool(np.array_equal(xb, xp))
    (ms_b, ms_p), (nverts, mism) = combine_over_ranks([ms_b, ms_p], [float(b.num_verts), 0.0 if same else 1.0],
                                                      dist, f"cuda:{local}")
    units = nverts * iters * K
    allm = meshgen.concat(meshes)
    peak, peak_kind = measured_peaks()
    step_s = ms_b / K * 1e-3
    achieved = sw_bytes / step_s / 1e9 if sw_bytes else None
    roofline = {
        "bound": "hbm",
        "kernel": "vbd::k_sweep (colour sweeps of all meshes, one launch per colour)",
        "achieved": achieved,
        "peak": peak,
        "peak_source": peak_kind,
        "unit": "GB/s",
        "frac": achieved / peak if achieved else None,
        "alg_bytes_per_step": sw_bytes,
        "alg_bytes_per_vertex_iteration": sw_bytes / (b.num_verts * iters) if sw_bytes else None,
        "sweep_launches_per_step": int(sw_launches),
        "launch_us_in_timed_region": (ms_b / K * 1e3 / sw_launches) if sw_launches else None,
        "how": "this rank's algorithmic sweep bytes of one step (60 B per incidence + 96 B per swept vertex) over "
               "the timed region's device time per step; predictor and velocity kernels are charged to the sweeps",
        "isolated": {
            "achieved": sw_bytes / (sw_ms * 1e-3) / 1e9 if sw_ms else None,
            "launch_us": sw_ms * 1e3 / sw_launches if sw_launches else None,
            "how": "one CUDA event pair around every sweep launched on its own (no graph, no PDL overlap)",
        },
    }
    return {
        "workload": f"{len(meshes)} jittered grid blocks, dims U{{4..24}}^3 x 6 tets, E log-U[1e4,1e6], "
                    "nu U[0.2,0.45], one face pinned, dt 1/60, 20 iterations, Chebyshev 0.9 (assumed), seed 2024",
        "meshes": len(meshes),
        "vertices": allm.num_verts,
        "tets": allm.num_tets,
        "steps": K,
        "value": units / (ms_b * 1e-3),
        "plain_value": units / (ms_p * 1e-3),
        "unit": UNIT,
        "speedup_vs_plain": ms_p / ms_b,
        "ms_per_step": ms_b / K,
        "plain_ms_per_step": ms_p / K,
        "launches_per_step": int(launches_b),
        "plain_launches_per_step": int(launches_p),
        "bitwise_equal_to_plain": mism == 0.0,
        "lanes": int(batch_lanes),
        "layout": int(batch_layout),
        "autotuned": tuned,
        "sharding": f"whole meshes over {world} rank(s), balanced by tet count" if world > 1 else "single GPU",
        "roofline": roofline,
    }


def bench_beam(local, stream, autotune=True):
    """The plain beam (16x4x4 cells, 425 vertices): 100 steps x 20 iterations from rest, the
    reference's CPU-runnable configuration, through the C ABI; wall time around the steps (the
    positions stay on the device).  The launch configuration is the autotuner's (set-up)."""
    import torch

    from vbd_tetmesh_b200 import _capi, build_solver, meshgen

    m = meshgen.beam()
    st = meshgen.BEAM_SETTINGS
    with torch.cuda.stream(stream):
        s = build_solver(m, device=local, stream=stream.cuda_stream)
        tuned = s.autotune(st["dt"], iterations=st["iterations"], repeats=5) if autotune else None
        best = None
        for _ in range(3):
            s.set_positions(m.x)
            s.set_velocities(m.v)
            s.sync()
            t0 = time.perf_counter()
            for _ in range(st["steps"]):
                s.step(st["dt"], st["iterations"], st["gravity"], True, st["rho"])
            s.sync()
            t = time.perf_counter() - t0
            best = t if best is None else min(best, t)
        launches_before = s.kernel_launches()
        s.step(st["dt"], st["iterations"], st["gravity"], True, st["rho"])
        s.sync()
        launches = s.kernel_launches() - launches_before
        persistent = s.get_option(_capi.OPT_PERSISTENT)
        path = {0: "captured CUDA graph", 1: "persistent kernel with grid barriers",
                2: "cluster walk (one thread-block cluster, positions in distributed shared memory)"}[persistent]
        graph_ms = None
        if persistent:  # the same shape through the captured graph of per-colour launches
            s.set_option(_capi.OPT_PERSISTENT, 0)
            s.set_positions(m.x)
            s.set_velocities(m.v)
            s.step(st["dt"], st["iterations"], st["gravity"], True, st["rho"])  # capture
            s.set_positions(m.x)
            s.set_velocities(m.v)
            s.sync()
            t0 = time.perf_counter()
            for _ in range(st["steps"]):
                s.step(st["dt"], st["iterations"], st["gravity"], True, st["rho"])
            s.sync()
            graph_ms = (time.perf_counter() - t0) * 1e3 / st["steps"]
        s.close()
    vi = m.num_verts * st["iterations"] * st["steps"]
    return {
        "workload": "beam 16x4x4 cells x 6 tets (425 vertices, 1,536 tets), E 1e5, nu 0.3, 100 steps x 20 "
                    "iterations, dt 1/60, Chebyshev 0.95, from rest",
        "ms_per_step": best * 1e3 / st["steps"],
        "value": vi / best,
        "unit": "vertex-iterations/s",
        "kernel_launches_per_step": launches,
        "path": path,
        "same_shape_captured_graph_ms_per_step": graph_ms,
        "autotuned": tuned,
        "how": "wall time around 100 vbd_solver_step calls (best of 3), positions resident on the device",
    }


def bench_adjoint(local, stream, autotune=True):
    """The differentiated configuration: 32x8x8 beam, per-tet materials, 30 steps x 30 iterations,
    checkpoint every 10 steps; forward (recorded) vs backward (recompute + implicit adjoint, 50
    Chebyshev-accelerated Gauss-Seidel sweeps per step), wall time around the C-ABI calls.  The
    launch configuration is the autotuner's (set-up)."""
    import torch

    from vbd_tetmesh_b200 import _capi, build_solver, meshgen

    m, tip, target = meshgen.diff_beam()
    st = meshgen.DIFF_SETTINGS
    with torch.cuda.stream(stream):
        s = build_solver(m, device=local, stream=stream.cuda_stream)
        tuned = s.autotune(st["dt"], iterations=st["iterations"], repeats=3) if autotune else None
        persistent = s.get_option(_capi.OPT_PERSISTENT)

        def forward_backward():
            res = []
            for _ in range(3):
                s.set_positions(m.x)
                s.set_velocities(m.v)
                s.record(st["checkpoint"])
                s.sync()
                t0 = time.perf_counter()
                for _ in range(st["steps"]):
                    s.step(st["dt"], st["iterations"], st["gravity"], True, st["rho"])
                s.sync()
                tf = time.perf_counter() - t0
                x = s.get_positions().astype(np.float64)
                g = np.zeros((m.num_verts, 3))
                g[tip] = 2.0 * (x[tip] - target)
                t0 = time.perf_counter()
                s.backward(g, None, st["adjoint_iterations"], st["adjoint_rho"])
                tb = time.perf_counter() - t0
                res.append((tf, tb))
            return min(res, key=lambda r: r[1])

        tf, tb = forward_backward()
        # the same shape through the captured graph of per-colour launches, for comparison
        graph = None
        if persistent:
            s.set_option(_capi.OPT_PERSISTENT, 0)
            gf, gb = forward_backward()
            graph = {"forward_ms": gf * 1e3, "backward_ms": gb * 1e3, "backward_over_forward": gb / gf}
        s.close()
    # Algorithmic bytes of the backward pass: the recomputed forward sweeps of the older segments
    # (the newest segment's states are kept) at the forward's 60 B per incidence + 96 B per swept
    # vertex, and the adjoint sweeps at 68 B per incidence (the record plus per-tet mu, lambda) +
    # 128 B per swept vertex (x, lambda read / write, G, y, lambda before the previous sweep).
    free = m.fixed == 0
    inc_free = int(free[m.tets].sum())
    nfree = int(free.sum())
    recomputed = st["steps"] - min(st["checkpoint"], st["steps"])
    fwd_iter = 60.0 * inc_free + 96.0 * nfree
    adj_sweep = 68.0 * inc_free + 128.0 * nfree
    alg = recomputed * st["iterations"] * fwd_iter + st["steps"] * st["adjoint_iterations"] * adj_sweep
    peak, peak_kind = measured_peaks()
    return {
        "workload": "32x8x8 beam x 6 tets (2,673 vertices, 12,288 tets), per-tet log-normal mu/lambda (sigma 0.2), "
                    "30 steps x 30 iterations, Chebyshev 0.95, checkpoint every 10 steps, loss on 25 tip vertices",
        "forward_ms": tf * 1e3,
        "backward_ms": tb * 1e3,
        "backward_over_forward": tb / tf,
        "adjoint_sweeps_per_step": st["adjoint_iterations"],
        "adjoint_rho": st["adjoint_rho"],
        "autotuned": tuned,
        "forward_path": {0: "captured CUDA graph", 1: "persistent kernel", 2: "cluster walk"}[persistent],
        "same_shape_captured_graph": graph,
        "accuracy": "checked in tests/test_gpu_adjoint.py: <= 1e-3 relative vs the FP64 implicit adjoint",
        "roofline": {
            "bound": "latency: 2,673 vertices give under 1% of the GPU's resident threads work",
            "achieved": alg / tb / 1e9,
            "peak": peak,
            "peak_source": peak_kind,
            "unit": "GB/s",
            "frac": alg / tb / 1e9 / peak,
            "alg_bytes_backward": alg,
            "how": "algorithmic bytes of the backward (recomputed forward sweeps + adjoint sweeps) over its wall "
                   "time around the C-ABI call (uploads and read-backs included)",
        },
    }


def bench_material_id(local, stream, autotune=True):
    """Batched material identification: 64 beams (Lx U{8..40}, Ly = Lz U{3..8}), hidden (E, nu) as the
    batched configuration, targets from a 20-step forward under gravity; per-mesh gradients of
    (log E, nu) from one batched forward + adjoint vs central finite differences of the batched
    forward (step 1e-2) at the initial guess, then 50 per-mesh trust-region iterations from E = 1e5,
    nu = 0.3."""
    import torch

    from vbd_tetmesh_b200 import material_id as mid

    FD_STEP = 1e-2  # the gradient check's finite-difference step (see "grad_fd")
    with torch.cuda.stream(stream):
        meshes, hidden = mid.beams(64)
        prob = mid.Problem.create(meshes, device=local, stream=stream.cuda_stream)
        targets = prob.forward(np.log(hidden[:, 0]), hidden[:, 1])
        st = mid.Settings()
        tuned = prob.solver.autotune(st.dt, iterations=st.iterations, repeats=2) if autotune else None
        logE0 = np.full(len(meshes), np.log(1e5))
        nu0 = np.full(len(meshes), 0.3)
        t0 = time.perf_counter()
        _, gE, gN = prob.loss_and_grad(logE0, nu0, targets)
        t_grad = time.perf_counter() - t0
        fE = prob.fd_grad(logE0, nu0, targets, "logE", FD_STEP)
        fN = prob.fd_grad(logE0, nu0, targets, "nu", FD_STEP)
        t0 = time.perf_counter()
        logE, nu, hist, final_losses, id_info = mid.identify(prob, targets, logE0, nu0, outer=50)
        t_id = time.perf_counter() - t0
        prob.solver.close()
    eE = np.abs(gE - fE) / np.maximum(np.abs(fE), 1e-30)
    eN = np.abs(gN - fN) / np.maximum(np.abs(fN), 1e-30)
    relE = np.abs(np.exp(logE) / hidden[:, 0] - 1.0)
    dnu = np.abs(nu - hidden[:, 1])
    q = lambda a: {"median": float(np.median(a)), "p90": float(np.percentile(a, 90)), "max": float(np.max(a))}  # noqa: E731
    return {
        "autotuned": tuned,
        "workload": f"{len(meshes)} beams, {prob.batch.num_verts} vertices, {prob.batch.num_tets} tets, "
                    f"{st.steps} steps x {st.iterations} iterations, adjoint {st.adjoint_iterations} sweeps, "
                    "all meshes in one solver",
        "gradient_seconds": t_grad,
        "grad_vs_fd_rel_logE": q(eE),
        "grad_vs_fd_rel_nu": q(eN),
        "grad_fd": "central differences of the batched FP32 GPU forward, step 1e-2 (in log E, and relative in nu); "
                   "below that the FP32 noise of the forward dominates: p90 of the nu error 5.1e-3 at step 1e-3, "
                   "2.2e-3 at 3e-3, 8.5e-4 at 1e-2, whether the adjoint runs 50 or 1,000 sweeps and the forward "
                   "100 or 1,000 iterations; checked against FP64 finite differences at converged iterations in "
                   "tests/test_gpu_material_id.py",
        "optimizer": "per-mesh trust-region descent on (log E, nu/0.1) with E kept in [5e3, 2e6] (the configuration "
                     "draws it from [1e4, 1e6]); every iteration is one batched forward + adjoint of all meshes; a mesh "
                     "steps by a 2x2 BFGS estimate from the adjoint's gradients until its trials fail twice in a row, or "
                     "its last 5 accepted steps together lowered its loss by less than 10% (the forward far from "
                     "converged, so the implicit gradient misleads); from then on it takes Levenberg-Marquardt steps "
                     "from the central-difference Jacobian of its final positions (four batched forwards)",
        "meshes_on_finite_differences": id_info["fd_meshes"],
        "batched_forward_adjoints": id_info["forward_backwards"],
        "batched_forwards": id_info["forwards"],
        "outer_iterations": 50,
        "identify_seconds": t_id,
        "loss_first": hist[0],
        "loss_last": hist[-1],
        "final_loss_per_mesh": q(np.asarray(final_losses)),
        "recovered_E_rel_err": q(relE),
        "recovered_nu_abs_err": q(dnu),
    }


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return

    import torch

    from vbd_tetmesh_b200 import _capi, build_solver, meshgen

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        dist = dist_mod

    mesh = meshgen.cube(args.cube)
    iters = args.iterations
    settings = meshgen.CUBE_SETTINGS
    dt, rho, grav = settings["dt"], settings["rho"], settings["gravity"]
    stream = torch.cuda.Stream(device=local)
    solver = build_solver(mesh, device=local, stream=stream.cuda_stream, lanes=args.lanes, layout=args.layout)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    # launch configuration picked by the project's autotuner (set-up, outside the timed region)
    tuned = None
    if not args.no_autotune:
        with torch.cuda.stream(stream):
            tuned = solver.autotune(dt, iterations=iters, repeats=3)
    if args.record_cache is not None:
        solver.set_option(_capi.OPT_RECORD_CACHE, args.record_cache)
    if args.persist_mb is not None:
        solver.set_option(_capi.OPT_RECORD_PERSIST_MB, args.persist_mb)
    if args.prefetch is not None:
        solver.set_option(_capi.OPT_PREFETCH, args.prefetch)
    if args.colour_lanes:
        solver.set_colour_lanes([int(v) for v in args.colour_lanes.split(",")])

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # nvidia-smi needs about a second to start sampling: launch it before the warm-up so that its
    # samples cover the timed passes
    clocks = ClockSampler(local, args.clocks_dir)
    clocks.start()
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            solver.step(dt, iters, grav, True, rho)
        solver.sync()
        clocks.wait_first_sample()

        # ---- timed region: device-resident steps, one event pair per step, L2 flushed between ----
        barrier()
        clocks.mark()
        launches0 = solver.kernel_launches()
        ms_total = 0.0
        torch.cuda.nvtx.range_push("timed")  # lets a profiler capture exactly these steps' kernels
        for _ in range(args.steps):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            solver.step(dt, iters, grav, True, rho)
            e1.record(stream)
            e1.synchronize()
            ms_total += e0.elapsed_time(e1)
        torch.cuda.nvtx.range_pop()
        barrier()
        launches = solver.kernel_launches() - launches0

        # ---- kernel timing pass: event pair around every colour-sweep launch ----
        solver.set_option(_capi.OPT_KERNEL_TIMING, 1)
        solver.kernel_time(reset=True)
        for _ in range(args.steps):
            flush.fill_(1.0)
            solver.step(dt, iters, grav, True, rho)
        sweep_ms, sweep_launches, sweep_bytes = solver.kernel_time(reset=True)
        solver.set_option(_capi.OPT_KERNEL_TIMING, 0)

        # ---- e2e: host buffers through the C ABI ----
        e2e_value = None
        h2d = d2h = 2 * 12 * mesh.num_verts
        if not args.no_e2e:
            xh = torch.empty((mesh.num_verts, 3), dtype=torch.float32, pin_memory=True).numpy()
            vh = torch.empty((mesh.num_verts, 3), dtype=torch.float32, pin_memory=True).numpy()
            solver.get_positions(xh)
            solver.get_velocities(vh)
            barrier()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                solver.set_positions(xh)
                solver.set_velocities(vh)
                solver.step(dt, iters, grav, True, rho)
                solver.get_positions(xh)
                solver.get_velocities(vh)
            e2e_s = time.perf_counter() - t0
            barrier()
        # clocks sampled over the three timed passes (device-resident, kernel-timed, e2e)
        clock_info = clocks.stop()

    sing, nonf = solver.status()
    from vbd_tetmesh_b200.sharding import combine_over_ranks

    (ms_max, e2e_max), _ = combine_over_ranks([ms_total, e2e_s if not args.no_e2e else 0.0], [], dist,
                                              f"cuda:{local}")
    units = float(mesh.num_verts) * iters * args.steps * world
    value = units / (ms_max * 1e-3)
    if not args.no_e2e:
        e2e_value = units / e2e_max

    peak, peak_kind = measured_peaks()
    # The sweep kernel's average launch duration in the timed region: the region's time (CUDA events
    # on the solver's stream, max over ranks) over the sweep launches in it.  The predictor and
    # velocity kernels (2 of 402 launches, 0.3% of the step's device time in the ncu launch list)
    # are charged to the sweeps, so this bounds the sweep's bandwidth from below.  The second pass,
    # one event pair around every sweep launched on its own (no graph, no PDL overlap), is reported
    # beside it as "isolated".
    achieved = iso_achieved = launch_us = None
    if sweep_launches and sweep_ms > 0:
        bytes_per_launch = sweep_bytes / sweep_launches
        launch_us = ms_max * 1e3 / sweep_launches
        achieved = bytes_per_launch / (launch_us * 1e-6) / 1e9
        iso_achieved = sweep_bytes / (sweep_ms * 1e-3) / 1e9
    # DRAM traffic per launch: the ncu-measured traffic / algorithmic-bytes ratio of the sweep
    # kernel (profiles/sweep_cube64_dram.txt) times this run's algorithmic bytes per launch
    traffic = None
    prof = os.path.join(ROOT, "profiles", "sweep_cube64_dram.txt")
    if os.path.exists(prof) and sweep_launches:
        for line in open(prof):
            if line.startswith("dram_traffic_over_algorithmic"):
                traffic = float(line.split("=")[1].split()[0]) * sweep_bytes / sweep_launches
    alg_bytes_per_vi = None
    if sweep_launches:
        alg_bytes_per_vi = sweep_bytes / (mesh.num_verts * iters * args.steps)

    result = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": dict(workload_config(mesh, iters), parallelism=f"replicas x{world}" if world > 1 else "single GPU",
                       lanes=solver.get_option(_capi.OPT_LANES), layout=solver.get_option(_capi.OPT_LAYOUT),
                       graph=solver.get_option(_capi.OPT_GRAPH), autotuned=tuned,
                       colour_lanes=solver.get_colour_lanes().tolist(),
                       record_cache=solver.get_option(_capi.OPT_RECORD_CACHE),
                       persist_mb=solver.get_option(_capi.OPT_RECORD_PERSIST_MB),
                       prefetch=solver.get_option(_capi.OPT_PREFETCH),
                       persistent=solver.get_option(_capi.OPT_PERSISTENT)),
        "gpu_launches": int(launches),
        "roofline": {
            "bound": "hbm",
            "kernel": "vbd::k_sweep (colour sweep)",
            "achieved": achieved,
            "peak": peak,
            "peak_source": peak_kind,
            "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None,
            "traffic": traffic,
            "sweep_launches_timed": int(sweep_launches),
            "launch_us_in_timed_region": launch_us,
            "alg_bytes_per_launch": (sweep_bytes / sweep_launches) if sweep_launches else None,
            "isolated": {
                "achieved": iso_achieved,
                "frac": (iso_achieved / peak) if iso_achieved else None,
                "launch_us": (sweep_ms * 1e3 / sweep_launches) if sweep_launches else None,
                "how": "one CUDA event pair around every sweep launched on its own (no graph, no PDL overlap)",
            },
            "alg_bytes_per_vertex_iteration": alg_bytes_per_vi,
            "step_frac_of_roofline": (value / world) * (alg_bytes_per_vi or 0) / (peak * 1e9),
        },
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "status": {"singular_skips": sing, "nonfinite": nonf},
    }
    if clock_info:
        result["clocks"] = clock_info
    if rank == 0:
        result["wrapper_semantics"] = bench_wrapper(mesh, local, stream)
    if not args.no_batched:
        result["batched"] = bench_batched(args, rank, world, local, stream, dist, barrier)
    if not args.no_adjoint and rank == 0:
        result["beam"] = bench_beam(local, stream, not args.no_autotune)
        result["adjoint"] = bench_adjoint(local, stream, not args.no_autotune)
    if not args.no_material_id and rank == 0:
        result["material_id"] = bench_material_id(local, stream, not args.no_autotune)

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu_value, cores, total, kind, what = cpu_reference(mesh, 3, warmup=1)
        result["cpu_baseline"] = {
            "value": cpu_value,
            "unit": UNIT,
            "cores": cores,
            "kind": kind,
            "sample": f"3 samples of 1 cube iteration (274,625 vertices, after 1 warm-up): {what}; its colour loop "
                      "runs one colour per thread, so at most 8 threads (the cube's 8 colours) are busy",
            "restatement": cpu_restatement(mesh),
        }
    solver.close()
    if rank == 0:
        print(json.dumps(result), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
