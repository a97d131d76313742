"""Python-side view of the C ABI: mesh set-up helpers and the GPU solver handle.

Names mirror the reference's C++ API (``VBD_GPU_Solver`` in VBD_GPU_Wrapper.h:7-45 and the step
loop of ``VBDsolver`` in VBD.cpp:60-112).  All compute runs in libvbd_b200.so; this module only
marshals arrays.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import call


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f32(a, shape=None) -> np.ndarray:
    out = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None:
        out = out.reshape(shape)
    return out


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def color_vertices(num_verts: int, tets: np.ndarray):
    """Greedy colouring (GraphColoring::colorVertices, GraphColoring.cpp:28-66).

    Returns (colour_of[N] int32, group_offsets[C+1] int32, group_vertices[N] int32)."""
    tets = _i32(tets)
    n, t = int(num_verts), int(tets.shape[0])
    colour_of = np.empty(n, np.int32)
    nc = C.c_int32(0)
    call("vbd_color_vertices", n, t, _ptr(tets), _ptr(colour_of), C.byref(nc), 0, None, None)
    offs = np.empty(nc.value + 1, np.int32)
    verts = np.empty(n, np.int32)
    call("vbd_color_vertices", n, t, _ptr(tets), _ptr(colour_of), C.byref(nc), nc.value, _ptr(offs), _ptr(verts))
    return colour_of, offs, verts


def mesh_mass(rest: np.ndarray, tets: np.ndarray, density: float):
    """Lumped masses and rest volumes (TetMesh::initialize, TetMesh.h:249-265)."""
    rest = _f32(rest, (-1, 3))
    tets = _i32(tets)
    n, t = rest.shape[0], tets.shape[0]
    mass = np.empty(n, np.float32)
    vol = np.empty(t, np.float32)
    call("vbd_mesh_mass", n, t, _ptr(rest), _ptr(tets), float(density), _ptr(mass), _ptr(vol))
    return mass, vol


def precompute_tets(rest: np.ndarray, tets: np.ndarray):
    """Dm^-1 (T,3,3) and V0 (T,) of the rest shape (VBDsolver::precomputeTetData, VBD.cpp:36-58)."""
    rest = _f32(rest, (-1, 3))
    tets = _i32(tets)
    n, t = rest.shape[0], tets.shape[0]
    dminv = np.empty((t, 3, 3), np.float32)
    v0 = np.empty(t, np.float32)
    call("vbd_precompute_tets", n, t, _ptr(rest), _ptr(tets), _ptr(dminv), _ptr(v0))
    return dminv, v0


def factored_record_error(dm_inv: np.ndarray):
    """(layout 3, layout 4) worst relative FP32 error of det M in the factored records, and the fraction
    of incidences on which layout 4 loses accuracy (above 1e-3: the automatic choice takes layout 3)."""
    d = _f32(dm_inv, (-1, 9))
    e3, e4, x4 = C.c_double(0.0), C.c_double(0.0), C.c_double(0.0)
    call("vbd_factored_record_error", int(d.shape[0]), _ptr(d), C.byref(e3), C.byref(e4), C.byref(x4))
    return e3.value, e4.value, x4.value


class GPUSolver:
    """One mesh (or batch of meshes) resident on one B200; wraps a ``vbd_solver*`` handle.

    Array arguments may be numpy arrays (host) or integer device pointers (``int``), e.g. a torch
    tensor's ``data_ptr()``; the library copies with unified addressing."""

    def __init__(self, device: int = 0, stream: int | None = None):
        h = C.c_void_p()
        call("vbd_solver_create", C.byref(h), int(device), None if stream is None else C.c_void_p(stream))
        self._h = h
        self.num_verts = 0
        self.num_tets = 0

    # -- lifetime ------------------------------------------------------------------------------
    def close(self) -> None:
        if self._h:
            call("vbd_solver_destroy", self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- set-up (VBD_GPU_Solver::initFromCPU, VBD_GPU_Wrapper.cu:246-315) -----------------------
    def init_from_cpu(self, positions, vertex_mass, fixed, tets, group_offsets, group_vertices, dm_inv, rest_vol,
                      tet_mu=None, tet_lambda=None, velocities=None, inertia=None) -> None:
        positions = _f32(positions, (-1, 3))
        n = positions.shape[0]
        tets = _i32(tets).reshape(-1, 4)
        t = tets.shape[0]
        args = [
            _ptr(positions),
            _ptr(None if velocities is None else _f32(velocities, (-1, 3))),
            _ptr(None if inertia is None else _f32(inertia, (-1, 3))),
            _ptr(_f32(vertex_mass)),
            _ptr(np.ascontiguousarray(fixed, dtype=np.uint8)),
            _ptr(tets),
            int(len(group_offsets) - 1),
            _ptr(_i32(group_offsets)),
            _ptr(_i32(group_vertices)),
            _ptr(_f32(dm_inv, (-1, 9))),
            _ptr(_f32(rest_vol)),
            _ptr(None if tet_mu is None else _f32(tet_mu)),
            _ptr(None if tet_lambda is None else _f32(tet_lambda)),
        ]
        # keep the converted arrays alive across the call
        self._keep = [positions, tets]
        call("vbd_solver_init", self._h, n, t, *args)
        self.num_verts, self.num_tets = n, t

    def set_materials(self, tet_mu=None, tet_lambda=None) -> None:
        call("vbd_solver_set_materials", self._h, _ptr(None if tet_mu is None else _f32(tet_mu)),
             _ptr(None if tet_lambda is None else _f32(tet_lambda)))

    def set_uniform_material(self, mu: float, lam: float) -> None:
        call("vbd_solver_set_uniform_material", self._h, float(mu), float(lam))

    # -- state transfer --------------------------------------------------------------------------
    def _set(self, name, a):
        if isinstance(a, int):
            call(name, self._h, C.c_void_p(a))
        else:
            a = _f32(a, (-1, 3))
            call(name, self._h, _ptr(a))

    def _get(self, name, out=None):
        if isinstance(out, int):
            call(name, self._h, C.c_void_p(out))
            return out
        if out is None:
            out = np.empty((self.num_verts, 3), np.float32)
        call(name, self._h, _ptr(out))
        return out

    def set_positions(self, a):
        self._set("vbd_solver_set_positions", a)

    def get_positions(self, out=None):
        return self._get("vbd_solver_get_positions", out)

    def set_velocities(self, a):
        self._set("vbd_solver_set_velocities", a)

    def get_velocities(self, out=None):
        return self._get("vbd_solver_get_velocities", out)

    def update_inertia_from_cpu(self, a):
        self._set("vbd_solver_set_inertia", a)

    def get_inertia(self, out=None):
        return self._get("vbd_solver_get_inertia", out)

    # -- solve ------------------------------------------------------------------------------------
    def solve_vbd(self, iterations: int, dt_sqr_reciprocal: float, use_acceleration: bool = True,
                  rho: float = 0.99, init_mode: int = _capi.INIT_FROM_INERTIA) -> None:
        call("vbd_solver_solve", self._h, int(iterations), float(dt_sqr_reciprocal), int(bool(use_acceleration)),
             float(rho), int(init_mode))

    def solve_iteration(self, dt_sqr_reciprocal: float) -> None:
        call("vbd_solver_solve_iteration", self._h, float(dt_sqr_reciprocal))

    def step(self, dt: float, iterations: int, gravity=(0.0, -9.8, 0.0), use_acceleration: bool = False,
             rho: float = 0.75, substeps: int = 1) -> None:
        g = np.asarray(gravity, dtype=np.float32)
        call("vbd_solver_step", self._h, float(dt), int(substeps), int(iterations), _ptr(g),
             int(bool(use_acceleration)), float(rho))

    def sync(self) -> None:
        call("vbd_solver_sync", self._h)

    # -- adjoint ----------------------------------------------------------------------------------
    def record(self, checkpoint_every: int = 10) -> None:
        """Start (k > 0) or stop (0) recording steps for the backward pass."""
        call("vbd_solver_record", self._h, int(checkpoint_every))

    def backward(self, dl_dx, dl_dv=None, adjoint_iterations: int = 50, adjoint_rho: float = 0.0):
        """Gradients of a final-state loss through the recorded steps:
        returns (dL/dx0 (N,3), dL/dv0 (N,3), dL/dmu (T,), dL/dlambda (T,))."""
        dl_dx = _f32(dl_dx, (-1, 3))
        dv = None if dl_dv is None else _f32(dl_dv, (-1, 3))
        gx = np.empty((self.num_verts, 3), np.float32)
        gv = np.empty((self.num_verts, 3), np.float32)
        gm = np.empty(self.num_tets, np.float32)
        gl = np.empty(self.num_tets, np.float32)
        call("vbd_solver_backward", self._h, _ptr(dl_dx), _ptr(dv), int(adjoint_iterations), float(adjoint_rho),
             _ptr(gx), _ptr(gv), _ptr(gm), _ptr(gl))
        return gx, gv, gm, gl

    # -- diagnostics ------------------------------------------------------------------------------
    def energy(self, kind: int, h: float = 1.0) -> float:
        out = C.c_double(0.0)
        call("vbd_solver_energy", self._h, int(kind), float(h), C.byref(out))
        return out.value

    def energy_history(self, reset: bool = True) -> np.ndarray:
        """The energies vbd_solver_step appended under OPT_ENERGY_EVERY (oldest first)."""
        n = C.c_int32(0)
        call("vbd_solver_energy_history", self._h, None, 0, C.byref(n), 0)
        out = np.empty(n.value, np.float64)
        call("vbd_solver_energy_history", self._h, _ptr(out), n.value, C.byref(n), int(bool(reset)))
        return out

    def status(self, reset: bool = False):
        sing = C.c_int64(0)
        nonf = C.c_int32(0)
        call("vbd_solver_status", self._h, C.byref(sing), C.byref(nonf), int(bool(reset)))
        return sing.value, bool(nonf.value)

    def set_option(self, option: int, value: int) -> None:
        call("vbd_solver_set_option", self._h, int(option), int(value))

    def get_option(self, option: int) -> int:
        v = C.c_int32(0)
        call("vbd_solver_get_option", self._h, int(option), C.byref(v))
        return v.value

    def set_colour_lanes(self, lanes=None) -> None:
        """Threads per vertex for each colour (None: VBD_OPT_LANES for every colour)."""
        if lanes is None:
            call("vbd_solver_set_colour_lanes", self._h, 0, None)
            return
        arr = _i32(lanes)
        call("vbd_solver_set_colour_lanes", self._h, int(arr.shape[0]), _ptr(arr))

    def get_colour_lanes(self) -> np.ndarray:
        nc = C.c_int32(0)
        call("vbd_solver_info", self._h, None, None, C.byref(nc))
        out = np.empty(nc.value, np.int32)
        call("vbd_solver_get_colour_lanes", self._h, nc.value, _ptr(out))
        return out

    def kernel_time(self, reset: bool = False):
        """(summed sweep-kernel ms, sweep launches, algorithmic bytes) timed since the last reset."""
        ms = C.c_double(0.0)
        n = C.c_int64(0)
        b = C.c_double(0.0)
        call("vbd_solver_kernel_time", self._h, C.byref(ms), C.byref(n), C.byref(b), int(bool(reset)))
        return ms.value, n.value, b.value

    def autotune(self, dt: float, iterations: int = 10, repeats: int = 2) -> dict:
        """Times the candidate launch configurations, keeps the fastest and restores the state."""
        out = (C.c_int32 * 5)()
        call("vbd_solver_autotune", self._h, float(dt), int(iterations), int(repeats), C.cast(out, C.c_void_p))
        res = dict(zip(("lanes", "layout", "prefetch", "pdl", "block"), list(out)))
        res["record_cache"] = self.get_option(_capi.OPT_RECORD_CACHE)
        res["persistent"] = self.get_option(_capi.OPT_PERSISTENT)
        res["colour_lanes"] = self.get_colour_lanes().tolist()
        if res["persistent"] == 2:
            res["cluster_ctas"] = self.get_option(_capi.OPT_CLUSTER_CTAS)
        return res

    def kernel_launches(self) -> int:
        v = C.c_int64(0)
        call("vbd_solver_kernel_launches", self._h, C.byref(v))
        return v.value


def build_solver(mesh, device: int = 0, stream: int | None = None, lanes: int | None = None,
                 layout: int | None = None, graph: bool | None = None) -> GPUSolver:
    """Colouring, masses and rest-shape data on the host, then one upload: the set-up sequence of
    the reference's driver (main.cpp:200-208) for a ``meshgen.Mesh``."""
    _, offs, verts = color_vertices(mesh.num_verts, mesh.tets)
    mass, _ = mesh_mass(mesh.rest, mesh.tets, mesh.density)
    dminv, v0 = precompute_tets(mesh.rest, mesh.tets)
    s = GPUSolver(device, stream)
    if lanes is not None:
        s.set_option(_capi.OPT_LANES, lanes)
    if layout is not None:
        s.set_option(_capi.OPT_LAYOUT, layout)
    if graph is not None:
        s.set_option(_capi.OPT_GRAPH, int(graph))
    s.init_from_cpu(mesh.x, mass, mesh.fixed, mesh.tets, offs, verts, dminv, v0, mesh.mu, mesh.lam,
                    velocities=mesh.v)
    s.vertex_mass = mass
    s.colour_groups = (offs, verts)
    return s


def build_batch_solver(batch, device: int = 0, stream: int | None = None) -> GPUSolver:
    """One solver for a meshgen.Batch: per-mesh masses and rest-shape data on the host, then
    vbd_solver_init_batch (per-mesh greedy colouring; colour c of all meshes in one launch)."""
    mass = np.concatenate([mesh_mass(m.rest, m.tets, m.density)[0] for m in batch.meshes])
    pre = [precompute_tets(m.rest, m.tets) for m in batch.meshes]
    dminv = np.concatenate([p[0] for p in pre])
    v0 = np.concatenate([p[1] for p in pre])
    s = GPUSolver(device, stream)
    keep = [np.ascontiguousarray(a) for a in (batch.vert_offsets, batch.tet_offsets)]
    arrs = [_f32(batch.x, (-1, 3)), _f32(batch.v, (-1, 3)), _f32(mass), np.ascontiguousarray(batch.fixed, np.uint8),
            _i32(batch.tets_local), _f32(dminv, (-1, 9)), _f32(v0), _f32(batch.mu), _f32(batch.lam)]
    call("vbd_solver_init_batch", s._h, len(batch.meshes), _ptr(_i32(keep[0])), _ptr(_i32(keep[1])),
         *[_ptr(a) for a in arrs])
    s.num_verts, s.num_tets = batch.num_verts, batch.num_tets
    s.vertex_mass = mass
    return s
