"""B200-native (sm_100a) Vertex Block Descent solver for tetrahedral Neo-Hookean elastodynamics.

The compute path is libvbd_b200.so (hand-written CUDA kernels behind a C ABI, include/vbd_b200.h);
this package only loads it and marshals arrays.  There is no CPU fallback: without the built
library, or without a B200, the solver calls raise.
"""
from ._capi import VBDError, lib  # noqa: F401
from .solver import GPUSolver, build_batch_solver, build_solver, color_vertices, mesh_mass, precompute_tets  # noqa: F401
from . import meshgen, surface, tetgen  # noqa: F401

__all__ = ["VBDError", "lib", "GPUSolver", "build_solver", "build_batch_solver", "color_vertices", "mesh_mass", "precompute_tets",
           "meshgen", "surface", "tetgen"]
