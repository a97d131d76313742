"""ctypes binding of libvbd_b200.so (the C ABI declared in include/vbd_b200.h).

The shared library is built in-tree by ``__graft_entry__.build()`` (``make -C
vbd_tetmesh_b200/csrc``).  Loading it never falls back to anything else: a missing library
raises ``OSError`` with the build command to run.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libvbd_b200.so")

VBD_OK = 0
STATUS_NAMES = {
    0: "VBD_OK",
    1: "VBD_ERR_INVALID_ARG",
    2: "VBD_ERR_CUDA",
    3: "VBD_ERR_STATE",
    4: "VBD_ERR_NONFINITE",
    5: "VBD_ERR_NO_DEVICE",
    6: "VBD_ERR_TIMEOUT",
    7: "VBD_ERR_ALLOC",
}
INIT_FROM_POSITIONS = 0
INIT_FROM_INERTIA = 1
ENERGY_IP = 0
ENERGY_ELASTIC_LOGJ = 1
ENERGY_RESIDUAL = 2
OPT_LANES = 0
OPT_LAYOUT = 1
OPT_GRAPH = 2
OPT_KERNEL_TIMING = 3
OPT_PREFETCH = 4
OPT_PDL = 5
OPT_BLOCK = 6
OPT_PERSISTENT = 7
OPT_ADJOINT_ALTERNATE = 8
OPT_SEMANTICS = 9
OPT_L2_PREFETCH = 10
OPT_RECORD_CACHE = 11
OPT_RECORD_PERSIST_MB = 12
OPT_ENERGY_EVERY = 13
OPT_CLUSTER_CTAS = 14
OPT_CLUSTER_RESIDENT = 15
SEMANTICS_VBDSOLVER = 0
SEMANTICS_GPU_WRAPPER = 1

_p = C.c_void_p
_i32 = C.c_int32
_f32 = C.c_float
_PI32 = C.POINTER(C.c_int32)
_PI64 = C.POINTER(C.c_int64)
_PF64 = C.POINTER(C.c_double)

# name -> argument types (every function returns int status, except the two noted)
SIGNATURES = {
    "vbd_version": [],
    "vbd_last_error": [],
    "vbd_color_vertices": [_i32, _i32, _p, _p, _PI32, _i32, _p, _p],
    "vbd_mesh_mass": [_i32, _i32, _p, _p, _f32, _p, _p],
    "vbd_precompute_tets": [_i32, _i32, _p, _p, _p, _p],
    "vbd_factored_record_error": [_i32, _p, _PF64, _PF64, _PF64],
    "vbd_tetgen_read_node": [C.c_char_p, _PI32, _PI32, _p, _i32],
    "vbd_tetgen_read_ele": [C.c_char_p, _i32, _i32, _PI32, _p, _i32],
    "vbd_pin_low_fraction": [_i32, _p, _i32, _f32, _p],
    "vbd_solver_create": [C.POINTER(_p), C.c_int, _p],
    "vbd_solver_destroy": [_p],
    "vbd_solver_init": [_p, _i32, _i32, _p, _p, _p, _p, _p, _p, _i32, _p, _p, _p, _p, _p, _p],
    "vbd_solver_init_batch": [_p, _i32, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p],
    "vbd_solver_set_materials": [_p, _p, _p],
    "vbd_solver_set_uniform_material": [_p, _f32, _f32],
    "vbd_solver_set_positions": [_p, _p],
    "vbd_solver_get_positions": [_p, _p],
    "vbd_solver_set_velocities": [_p, _p],
    "vbd_solver_get_velocities": [_p, _p],
    "vbd_solver_set_inertia": [_p, _p],
    "vbd_solver_get_inertia": [_p, _p],
    "vbd_solver_solve": [_p, _i32, _f32, _i32, _f32, _i32],
    "vbd_solver_solve_iteration": [_p, _f32],
    "vbd_solver_step": [_p, _f32, _i32, _i32, _p, _i32, _f32],
    "vbd_solver_sync": [_p],
    "vbd_solver_record": [_p, _i32],
    "vbd_solver_backward": [_p, _p, _p, _i32, _f32, _p, _p, _p, _p],
    "vbd_solver_energy": [_p, _i32, _f32, _PF64],
    "vbd_solver_energy_history": [_p, _p, _i32, _PI32, _i32],
    "vbd_solver_status": [_p, _PI64, _PI32, _i32],
    "vbd_solver_set_option": [_p, _i32, _i32],
    "vbd_solver_get_option": [_p, _i32, _PI32],
    "vbd_solver_info": [_p, _PI32, _PI32, _PI32],
    "vbd_solver_set_colour_lanes": [_p, _i32, _p],
    "vbd_solver_get_colour_lanes": [_p, _i32, _p],
    "vbd_solver_kernel_launches": [_p, _PI64],
    "vbd_solver_kernel_time": [_p, _PF64, _PI64, _PF64, _i32],
    "vbd_solver_autotune": [_p, _f32, _i32, _i32, _p],
    "vbd_solver_barrier_selftest": [_p, C.c_int64, _PI32],
    "vbd_ip_energy_noalloc": [_i32, _i32, _p, _p, _p, _p, _p, _p, _p, _p, _f32, _p, _p],
}

_lib = None


class VBDError(RuntimeError):
    """A C-ABI call returned a non-zero vbd_status."""

    def __init__(self, func: str, code: int, message: str):
        self.func = func
        self.code = code
        self.message = message
        super().__init__(f"{func} -> {STATUS_NAMES.get(code, code)}: {message}")


def lib() -> C.CDLL:
    """Loads libvbd_b200.so once and declares every C-ABI signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing: build it with `make -C {os.path.join(_HERE, 'csrc')}`")
    L = C.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_char_p if name == "vbd_last_error" else C.c_int
    _lib = L
    return L


def check(func: str, code: int) -> None:
    if code != VBD_OK:
        msg = lib().vbd_last_error().decode(errors="replace")
        raise VBDError(func, code, msg)


def call(name: str, *args) -> None:
    """Calls a C-ABI function and raises VBDError on a non-zero status."""
    check(name, getattr(lib(), name)(*args))
