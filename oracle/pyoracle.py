"""ctypes wrapper of the oracle (oracle/libvbd_oracle.so) -- TEST INFRASTRUCTURE ONLY.

The oracle restates the reference's CPU VBD path (see the header of vbd_oracle.cpp for the
file:line map).  Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module, and only as the checker / the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libvbd_oracle.so")
_lib = None

LITERAL, LITERAL_FULL12, CLOSED, WRAPPER = 0, 1, 2, 3

_p = C.c_void_p
_i = C.c_int
_d = C.c_double


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", _HERE], check=True, capture_output=True)
        L = C.CDLL(LIB_PATH)
        L.orc_color_vertices.argtypes = [_i, _i, _p, _p]
        L.orc_color_vertices.restype = _i
        L.orc_mesh_setup.argtypes = [_i, _i, _i, _p, _p, _d, _p, _p, _p, _p]
        L.orc_mesh_setup.restype = None
        L.orc_simulate.argtypes = [_i, _i, _i, _i, _i, _p, _p, _p, _p, _p, _p, _p, _d, _d, _i, _i, _p, _i, _d, _i,
                                   _p, _p, _p, _p, _p]
        L.orc_simulate.restype = _i
        L.orc_solve.argtypes = [_i, _i, _i, _i, _i, _p, _p, _p, _p, _p, _p, _p, _d, _d, _i, _i, _d, _i, _p]
        L.orc_solve.restype = _i
        L.orc_residual.argtypes = [_i, _i, _p, _p, _p, _p, _p, _p, _p, _d, _d]
        L.orc_residual.restype = _d
        L.orc_tet_block.argtypes = [_i, _i, _p, _p, _d, _d, _d, _i, _p, _p]
        L.orc_tet_block.restype = None
        L.orc_ip_energy.argtypes = [_i, _i, _p, _p, _p, _p, _p, _p, _p, _p, _d]
        L.orc_ip_energy.restype = _d
        L.orc_handle_create.argtypes = [_i, _i, _i, _i, _p, _p, _p, _p, _p, _p, _p, _d]
        L.orc_handle_create.restype = _p
        L.orc_handle_step.argtypes = [_p, _i, _d, _i, _i, _p, _i, _d, _i]
        L.orc_handle_step.restype = None
        L.orc_handle_positions.argtypes = [_p, _p]
        L.orc_handle_positions.restype = None
        L.orc_handle_destroy.argtypes = [_p]
        L.orc_handle_destroy.restype = None
        L.orc_adjoint_f64.argtypes = [_i, _i, _p, _p, _p, _p, _p, _p, _p, _d, _d, _i, _p, _i, _d, _i, _p, _p, _p, _p,
                                       _p, _p, _p, _p]
        L.orc_adjoint_f64.restype = _i
        L.orc_num_threads_max.argtypes = []
        L.orc_num_threads_max.restype = _i
        _lib = L
    return _lib


def _d64(a, shape=None):
    out = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    return out if shape is None else out.reshape(shape)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def color_vertices(num_verts, tets):
    tets = np.ascontiguousarray(tets, dtype=np.int32)
    out = np.empty(num_verts, np.int32)
    nc = lib().orc_color_vertices(int(num_verts), int(tets.shape[0]), _ptr(tets), _ptr(out))
    return out, nc


def mesh_setup(rest, tets, density, precision=32):
    """(mass[N], tet_rest_vol[T], dminv[T,3,3], v0[T]) as TetMesh::initialize + precomputeTetData."""
    rest = _d64(rest, (-1, 3))
    tets = np.ascontiguousarray(tets, dtype=np.int32)
    n, t = rest.shape[0], tets.shape[0]
    mass = np.empty(n)
    trv = np.empty(t)
    dminv = np.empty((t, 3, 3))
    v0 = np.empty(t)
    lib().orc_mesh_setup(precision, n, t, _ptr(rest), _ptr(tets), float(density), _ptr(mass), _ptr(trv),
                         _ptr(dminv), _ptr(v0))
    return mass, trv, dminv, v0


def simulate(mesh, steps, dt, iterations, gravity=(0.0, -9.8, 0.0), use_acceleration=True, rho=0.95,
             substeps=1, precision=32, mode=LITERAL, threads=1, energy_history=False, x0=None, v0=None):
    """Runs ``steps`` calls of VBDsolver::step on a meshgen.Mesh.

    Returns dict(x=(N,3), v=(N,3), ip=(steps,), ehist=array|None, ncolors=int)."""
    rest = _d64(mesh.rest, (-1, 3))
    x = _d64(mesh.x if x0 is None else x0, (-1, 3))
    v = _d64(mesh.v if v0 is None else v0, (-1, 3))
    tets = np.ascontiguousarray(mesh.tets, dtype=np.int32)
    fixed = np.ascontiguousarray(mesh.fixed, dtype=np.uint8)
    mu, lam = _d64(mesh.mu), _d64(mesh.lam)
    n, t = rest.shape[0], tets.shape[0]
    g = _d64(gravity)
    xo = np.empty((n, 3))
    vo = np.empty((n, 3))
    ip = np.empty(max(steps, 1))
    per = substeps * ((iterations + 9) // 10)
    eh = np.empty(max(steps * per, 1)) if energy_history else None
    nc = C.c_int(0)
    lib().orc_simulate(precision, mode, threads, n, t, _ptr(rest), _ptr(x), _ptr(v), _ptr(tets), _ptr(fixed),
                       _ptr(mu), _ptr(lam), float(mesh.density), float(dt), int(substeps), int(iterations), _ptr(g),
                       int(bool(use_acceleration)), float(rho), int(steps), _ptr(xo), _ptr(vo), _ptr(ip),
                       _ptr(eh), C.byref(nc))
    return dict(x=xo, v=vo, ip=ip[:steps], ehist=eh, ncolors=nc.value)


def solve(mesh, x0, y0, dt_sqr_reciprocal, iterations, use_acceleration=True, rho=0.99, init_from_inertia=False,
          precision=32, mode=LITERAL, threads=1):
    rest = _d64(mesh.rest, (-1, 3))
    x0 = _d64(x0, (-1, 3))
    y0 = _d64(y0, (-1, 3))
    tets = np.ascontiguousarray(mesh.tets, dtype=np.int32)
    fixed = np.ascontiguousarray(mesh.fixed, dtype=np.uint8)
    mu, lam = _d64(mesh.mu), _d64(mesh.lam)
    n, t = rest.shape[0], tets.shape[0]
    out = np.empty((n, 3))
    lib().orc_solve(precision, mode, threads, n, t, _ptr(rest), _ptr(x0), _ptr(y0), _ptr(tets), _ptr(fixed),
                    _ptr(mu), _ptr(lam), float(mesh.density), float(dt_sqr_reciprocal), int(iterations),
                    int(bool(use_acceleration)), float(rho), int(bool(init_from_inertia)), _ptr(out))
    return out


def residual(mesh, x, y, dt_sqr_reciprocal):
    rest = _d64(mesh.rest, (-1, 3))
    tets = np.ascontiguousarray(mesh.tets, dtype=np.int32)
    fixed = np.ascontiguousarray(mesh.fixed, dtype=np.uint8)
    mu, lam = _d64(mesh.mu), _d64(mesh.lam)
    x, y = _d64(x, (-1, 3)), _d64(y, (-1, 3))
    return lib().orc_residual(rest.shape[0], tets.shape[0], _ptr(rest), _ptr(x), _ptr(y), _ptr(tets), _ptr(fixed),
                              _ptr(mu), _ptr(lam), float(mesh.density), float(dt_sqr_reciprocal))


def tet_block(F, dminv, mu, lam, vol, n, mode=LITERAL, precision=64):
    F = _d64(F, (3, 3))
    D = _d64(dminv, (3, 3))
    H = np.empty((3, 3))
    g = np.empty(3)
    lib().orc_tet_block(precision, mode, _ptr(F), _ptr(D), float(mu), float(lam), float(vol), int(n), _ptr(H),
                        _ptr(g))
    return H, g


def ip_energy(x, y, mass, tets, dminv, v0, mu, lam, h):
    x, y = _d64(x, (-1, 3)), _d64(y, (-1, 3))
    tets = np.ascontiguousarray(tets, dtype=np.int32)
    return lib().orc_ip_energy(x.shape[0], tets.shape[0], _ptr(x), _ptr(y), _ptr(_d64(mass)), _ptr(tets),
                               _ptr(_d64(dminv, (-1, 9))), _ptr(_d64(v0)), _ptr(_d64(mu)), _ptr(_d64(lam)),
                               float(h))


def adjoint_f64(mesh, steps, dt, iterations, dLdx_fn=None, gravity=(0.0, -9.8, 0.0), use_acceleration=True, rho=0.9,
                x0=None, v0=None, mu=None, lam=None):
    """FP64 forward (substeps 1) and implicit adjoint.  dLdx_fn(x_final) -> dL/dx_final (N,3).
    Returns dict(x=final positions, gx0, gv0, gmu, glam, cg_iterations, residual)."""
    rest = _d64(mesh.rest, (-1, 3))
    x = _d64(mesh.x if x0 is None else x0, (-1, 3))
    v = _d64(mesh.v if v0 is None else v0, (-1, 3))
    tets = np.ascontiguousarray(mesh.tets, dtype=np.int32)
    fixed = np.ascontiguousarray(mesh.fixed, dtype=np.uint8)
    mu = _d64(mesh.mu if mu is None else mu)
    lam = _d64(mesh.lam if lam is None else lam)
    n, t = rest.shape[0], tets.shape[0]
    g = _d64(gravity)
    xf = np.empty((n, 3))
    args = (n, t, _ptr(rest), _ptr(x), _ptr(v), _ptr(tets), _ptr(fixed), _ptr(mu), _ptr(lam), float(mesh.density),
            float(dt), int(iterations), _ptr(g), int(bool(use_acceleration)), float(rho), int(steps))
    if dLdx_fn is None:
        lib().orc_adjoint_f64(*args, None, None, _ptr(xf), None, None, None, None, None)
        return dict(x=xf)
    # forward once to get the final state, then again with the loss gradient
    lib().orc_adjoint_f64(*args, None, None, _ptr(xf), None, None, None, None, None)
    dl = _d64(dLdx_fn(xf), (-1, 3))
    gx0 = np.empty((n, 3))
    gv0 = np.empty((n, 3))
    gmu = np.empty(t)
    glam = np.empty(t)
    res = C.c_double(0.0)
    it = lib().orc_adjoint_f64(*args, _ptr(dl), None, _ptr(xf), _ptr(gx0), _ptr(gv0), _ptr(gmu), _ptr(glam),
                               C.byref(res))
    return dict(x=xf, gx0=gx0, gv0=gv0, gmu=gmu, glam=glam, cg_iterations=it, residual=res.value)


def max_threads():
    return lib().orc_num_threads_max()


class Handle:
    """A persistent FP32 oracle simulation (set-up once, then timed steps)."""

    def __init__(self, mesh, mode=LITERAL_FULL12, threads=1):
        self._keep = [_d64(mesh.rest, (-1, 3)), _d64(mesh.x, (-1, 3)), _d64(mesh.v, (-1, 3)),
                      np.ascontiguousarray(mesh.tets, dtype=np.int32), np.ascontiguousarray(mesh.fixed, np.uint8),
                      _d64(mesh.mu), _d64(mesh.lam)]
        r, x, v, t, f, mu, lam = self._keep
        self.n = r.shape[0]
        self._h = lib().orc_handle_create(mode, threads, r.shape[0], t.shape[0], _ptr(r), _ptr(x), _ptr(v), _ptr(t),
                                          _ptr(f), _ptr(mu), _ptr(lam), float(mesh.density))

    def step(self, steps, dt, iterations, gravity=(0.0, -9.8, 0.0), use_acceleration=True, rho=0.9, substeps=1,
             energy=True):
        g = _d64(gravity)
        lib().orc_handle_step(self._h, int(steps), float(dt), int(substeps), int(iterations), _ptr(g),
                              int(bool(use_acceleration)), float(rho), int(bool(energy)))

    def positions(self):
        out = np.empty((self.n, 3))
        lib().orc_handle_positions(self._h, _ptr(out))
        return out

    def close(self):
        if self._h:
            lib().orc_handle_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


# ---- the reference's own sources, compiled against the Eigen-API subset (oracle/_ref) -------------

REF_LIB_PATH = os.path.join(_HERE, "_ref", "libvbdref.so")
_ref_lib = None


def ref_available():
    return os.path.exists(REF_LIB_PATH)


def ref_lib():
    global _ref_lib
    if _ref_lib is None:
        L = C.CDLL(REF_LIB_PATH)
        f = C.c_float
        L.ref_create.argtypes = [_i, _i, _p, _p, _p, _p, _p, f, f, f, f, _i, _i, _p, _i, f, _i]
        L.ref_create.restype = _p
        L.ref_step.argtypes = [_p, _i]
        L.ref_step.restype = None
        L.ref_iterations.argtypes = [_p, _i]
        L.ref_iterations.restype = None
        L.ref_state.argtypes = [_p, _p, _p]
        L.ref_state.restype = None
        L.ref_setup.argtypes = [_p, _p, _p, _p, _p, _p]
        L.ref_setup.restype = _i
        L.ref_energy_history.argtypes = [_p, _p, _i]
        L.ref_energy_history.restype = _i
        L.ref_destroy.argtypes = [_p]
        L.ref_destroy.restype = None
        _ref_lib = L
    return _ref_lib


class RefHandle:
    """The reference's TetMesh + VBDsolver (scalar mu / lambda, as VBD.cpp:214-215 uses)."""

    def __init__(self, mesh, dt, iterations, gravity=(0.0, -9.8, 0.0), use_acceleration=True, rho=0.95,
                 substeps=1, threads=1):
        f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)
        self._keep = [f32(mesh.rest).reshape(-1, 3), f32(mesh.x).reshape(-1, 3), f32(mesh.v).reshape(-1, 3),
                      np.ascontiguousarray(mesh.tets, dtype=np.int32), np.ascontiguousarray(mesh.fixed, np.uint8),
                      f32(gravity)]
        r, x, v, t, fx, g = self._keep
        self.n, self.t = r.shape[0], t.shape[0]
        self._h = ref_lib().ref_create(self.n, self.t, _ptr(r), _ptr(x), _ptr(v), _ptr(t), _ptr(fx),
                                       float(mesh.density), float(mesh.mu[0]), float(mesh.lam[0]), float(dt),
                                       int(substeps), int(iterations), _ptr(g), int(bool(use_acceleration)),
                                       float(rho), int(threads))

    def step(self, n=1):
        ref_lib().ref_step(self._h, int(n))

    def iterations(self, n):
        ref_lib().ref_iterations(self._h, int(n))

    def state(self):
        x = np.empty((self.n, 3), np.float32)
        v = np.empty((self.n, 3), np.float32)
        ref_lib().ref_state(self._h, _ptr(x), _ptr(v))
        return x, v

    def setup(self):
        col = np.empty(self.n, np.int32)
        mass = np.empty(self.n, np.float32)
        trv = np.empty(self.t, np.float32)
        dm = np.empty((self.t, 3, 3), np.float32)
        v0 = np.empty(self.t, np.float32)
        nc = ref_lib().ref_setup(self._h, _ptr(col), _ptr(mass), _ptr(trv), _ptr(dm), _ptr(v0))
        return dict(colour_of=col, ncolours=nc, mass=mass, tet_rest_vol=trv, dminv=dm, v0=v0)

    def energy_history(self):
        n = ref_lib().ref_energy_history(self._h, None, 0)
        out = np.empty(max(n, 1))
        ref_lib().ref_energy_history(self._h, _ptr(out), n)
        return out[:n]

    def close(self):
        if self._h:
            ref_lib().ref_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


# ---- the reference's GPU wrapper (VBD_GPU_Solver), built by `make -C oracle refgpu` -------------
# Runs the reference's own kernels on a GPU; used to pin the wrapper-semantics restatement and to
# time the reference's GPU path.  Available only where oracle/_ref/libvbdref_gpu.so was built and
# a GPU is present.
REF_GPU_LIB_PATH = os.path.join(_HERE, "_ref", "libvbdref_gpu.so")
_ref_gpu_lib = None


def ref_gpu_available():
    return os.path.exists(REF_GPU_LIB_PATH)


def ref_gpu_lib():
    global _ref_gpu_lib
    if _ref_gpu_lib is None:
        L = C.CDLL(REF_GPU_LIB_PATH)
        f = C.c_float
        L.refgpu_create.argtypes = [_i, _i, _p, _p, _p, _p, f, f, f, f, _i, _i, _p, _i, f]
        L.refgpu_create.restype = _p
        L.refgpu_set_inertia.argtypes = [_p, _p]
        L.refgpu_set_inertia.restype = _i
        L.refgpu_solve.argtypes = [_p, _i, f, f, f, _i, f, _p]
        L.refgpu_solve.restype = _i
        L.refgpu_frame.argtypes = [_p, f, f]
        L.refgpu_frame.restype = _i
        L.refgpu_positions.argtypes = [_p, _p]
        L.refgpu_positions.restype = _i
        L.refgpu_velocities.argtypes = [_p, _p]
        L.refgpu_velocities.restype = None
        L.refgpu_destroy.argtypes = [_p]
        L.refgpu_destroy.restype = None
        _ref_gpu_lib = L
    return _ref_gpu_lib


class RefGpuHandle:
    """The reference's TetMesh + VBDsolver (colouring, Dm^-1, V0) + VBD_GPU_Solver on cuda:0, with
    scalar mu / lambda as main.cpp passes them."""

    def __init__(self, mesh, dt=1.0 / 60.0, iterations=20, gravity=(0.0, -9.8, 0.0), use_acceleration=True,
                 rho=0.95, substeps=1):
        f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
        self._keep = [f32(mesh.rest).reshape(-1, 3), f32(mesh.x).reshape(-1, 3),
                      np.ascontiguousarray(mesh.tets, dtype=np.int32), np.ascontiguousarray(mesh.fixed, np.uint8),
                      f32(gravity)]
        r, x, t, fx, g = self._keep
        self.n = r.shape[0]
        self.mu, self.lam = float(mesh.mu[0]), float(mesh.lam[0])
        self._h = ref_gpu_lib().refgpu_create(self.n, t.shape[0], _ptr(r), _ptr(x), _ptr(t), _ptr(fx),
                                              float(mesh.density), self.mu, self.lam, float(dt), int(substeps),
                                              int(iterations), _ptr(g), int(bool(use_acceleration)), float(rho))
        if not self._h:
            raise RuntimeError("the reference's VBD_GPU_Solver could not be set up")

    def set_inertia(self, y):
        y = np.ascontiguousarray(y, dtype=np.float32).reshape(-1, 3)
        if ref_gpu_lib().refgpu_set_inertia(self._h, _ptr(y)):
            raise RuntimeError("CUDA error in the reference's updateInertiaFromCPU")

    def solve(self, iterations, dt_sqr_reciprocal, use_acceleration=True, rho=0.99):
        """VBD_GPU_Solver::solveVBD; returns its device time in ms."""
        ms = C.c_float(0.0)
        if ref_gpu_lib().refgpu_solve(self._h, int(iterations), float(dt_sqr_reciprocal), self.mu, self.lam,
                                      int(bool(use_acceleration)), float(rho), C.byref(ms)):
            raise RuntimeError("CUDA error in the reference's solveVBD")
        return ms.value

    def frame(self, n=1):
        """n frames of main.cpp's GPU loop."""
        for _ in range(n):
            if ref_gpu_lib().refgpu_frame(self._h, self.mu, self.lam):
                raise RuntimeError("CUDA error in the reference's GPU loop")

    def positions(self):
        x = np.empty((self.n, 3), np.float32)
        if ref_gpu_lib().refgpu_positions(self._h, _ptr(x)):
            raise RuntimeError("CUDA error in the reference's copyPositionsToCPU")
        return x

    def velocities(self):
        v = np.empty((self.n, 3), np.float32)
        ref_gpu_lib().refgpu_velocities(self._h, _ptr(v))
        return v

    def close(self):
        if self._h:
            ref_gpu_lib().refgpu_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()
