"""Procedural tetrahedral meshes and the benchmark configurations of the VBD path.

Hex grids of ``lx x ly x lz`` cells, each cell split into 6 tets (Kuhn / Freudenthal split around
the 000 -> 111 diagonal; tet = path 000 -> e_a -> e_a + e_b -> 111 over the six axis orders, so
the triangulation is conforming).  Vertex id = i + (lx+1) (j + (ly+1) k): x fastest, which is the
order the greedy colouring sees.  Tet order: cells with i fastest, then the six axis orders
(0,1,2) (0,2,1) (1,0,2) (1,2,0) (2,0,1) (2,1,0).  All randomness comes from
``numpy.random.default_rng(seed)``.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

AXIS_ORDERS = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))


def lame(E: float, nu: float) -> tuple[float, float]:
    """(mu, lambda) of Young's modulus E and Poisson ratio nu."""
    return E / (2.0 * (1.0 + nu)), E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))


@dataclass
class Mesh:
    """A tet mesh plus its per-vertex / per-tet simulation inputs (float32 / int32)."""

    rest: np.ndarray            # (N, 3) float32 rest positions
    x: np.ndarray               # (N, 3) float32 current positions
    v: np.ndarray               # (N, 3) float32 velocities
    tets: np.ndarray            # (T, 4) int32
    fixed: np.ndarray           # (N,) uint8
    mu: np.ndarray              # (T,) float32
    lam: np.ndarray             # (T,) float32
    density: float = 1000.0
    ijk: np.ndarray | None = None  # (N, 3) int32 grid coordinates
    dims: tuple = ()
    meta: dict = field(default_factory=dict)

    @property
    def num_verts(self) -> int:
        return int(self.rest.shape[0])

    @property
    def num_tets(self) -> int:
        return int(self.tets.shape[0])

    def bbox_diag(self) -> float:
        lo, hi = self.x.min(0).astype(np.float64), self.x.max(0).astype(np.float64)
        return float(np.linalg.norm(hi - lo))


def grid(lx: int, ly: int, lz: int, cell: float, jitter: float = 0.0, seed: int = 0):
    """Vertices (float64, (N,3)), tets (int32, (T,4)) and grid coordinates of a Kuhn-split grid.

    ``jitter`` displaces every vertex by U(-jitter, jitter) * cell per component."""
    k, j, i = np.meshgrid(np.arange(lz + 1), np.arange(ly + 1), np.arange(lx + 1), indexing="ij")
    ijk = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.int32)
    pos = ijk.astype(np.float64) * cell
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        pos = pos + rng.uniform(-jitter, jitter, size=pos.shape) * cell
    ck, cj, ci = np.meshgrid(np.arange(lz), np.arange(ly), np.arange(lx), indexing="ij")
    base = (ci + (lx + 1) * (cj + (ly + 1) * ck)).ravel().astype(np.int64)
    step = np.array([1, lx + 1, (lx + 1) * (ly + 1)], dtype=np.int64)
    tets = np.empty((base.size, 6, 4), dtype=np.int64)
    for o, (a, b, _c) in enumerate(AXIS_ORDERS):
        tets[:, o, 0] = base
        tets[:, o, 1] = base + step[a]
        tets[:, o, 2] = base + step[a] + step[b]
        tets[:, o, 3] = base + step.sum()
    return pos, tets.reshape(-1, 4).astype(np.int32), ijk


def _finish(pos, tets, ijk, fixed, E, nu, density, v=None, dims=(), meta=None) -> Mesh:
    mu, lam = lame(E, nu)
    n, t = pos.shape[0], tets.shape[0]
    p32 = pos.astype(np.float32)
    return Mesh(
        rest=p32.copy(),
        x=p32.copy(),
        v=np.zeros((n, 3), np.float32) if v is None else v.astype(np.float32),
        tets=tets,
        fixed=fixed.astype(np.uint8),
        mu=np.full(t, mu, np.float32),
        lam=np.full(t, lam, np.float32),
        density=float(density),
        ijk=ijk,
        dims=dims,
        meta=dict(meta or {}),
    )


def beam(lx=16, ly=4, lz=4, cell=0.05, E=1e5, nu=0.3, density=1000.0, jitter=0.0, seed=0) -> Mesh:
    """Cantilever beam, x = 0 face pinned (16x4x4 cells: 425 vertices, 1,536 tets)."""
    pos, tets, ijk = grid(lx, ly, lz, cell, jitter, seed)
    return _finish(pos, tets, ijk, ijk[:, 0] == 0, E, nu, density, dims=(lx, ly, lz),
                   meta=dict(kind="beam", cell=cell, E=E, nu=nu, jitter=jitter, seed=seed))


def cube(n=64, E=1e6, nu=0.4, density=1000.0, jitter=0.2, seed=1234, vel_sigma=0.5) -> Mesh:
    """Jittered unit cube of n^3 cells (cell 1/n), bottom face (j = 0) pinned, initial velocities
    N(0, vel_sigma) per component on free vertices (64^3: 274,625 vertices, 1,572,864 tets)."""
    cell = 1.0 / n
    pos, tets, ijk = grid(n, n, n, cell, jitter, seed)
    fixed = ijk[:, 1] == 0
    rng = np.random.default_rng(seed + 1)
    v = rng.normal(0.0, vel_sigma, size=pos.shape)
    v[fixed] = 0.0
    return _finish(pos, tets, ijk, fixed, E, nu, density, v=v, dims=(n, n, n),
                   meta=dict(kind="cube", cell=cell, E=E, nu=nu, jitter=jitter, seed=seed, vel_sigma=vel_sigma))


def jittered_block(lx, ly, lz, cell=0.05, jitter=0.25, E=1e5, nu=0.3, density=1000.0, seed=0,
                   pin_face="x0", per_tet_sigma=0.0) -> Mesh:
    """A jittered grid block with one face pinned (x0, x1, y0, y1, z0, z1) and, optionally,
    per-tet log-normal perturbations of mu and lambda with standard deviation per_tet_sigma."""
    pos, tets, ijk = grid(lx, ly, lz, cell, jitter, seed)
    axis = "xyz".index(pin_face[0])
    hi = (lx, ly, lz)[axis]
    fixed = ijk[:, axis] == (0 if pin_face[1] == "0" else hi)
    m = _finish(pos, tets, ijk, fixed, E, nu, density, dims=(lx, ly, lz),
                meta=dict(kind="block", cell=cell, E=E, nu=nu, jitter=jitter, seed=seed, pin_face=pin_face))
    if per_tet_sigma > 0.0:
        rng = np.random.default_rng(seed + 7)
        t = m.num_tets
        m.mu = (m.mu.astype(np.float64) * np.exp(rng.normal(0.0, per_tet_sigma, t))).astype(np.float32)
        m.lam = (m.lam.astype(np.float64) * np.exp(rng.normal(0.0, per_tet_sigma, t))).astype(np.float32)
    return m


# Simulation settings of the configurations (dt, iterations, Chebyshev rho, steps, gravity).
BEAM_SETTINGS = dict(dt=1.0 / 60.0, iterations=20, rho=0.95, steps=100, gravity=(0.0, -9.8, 0.0))
CUBE_SETTINGS = dict(dt=1.0 / 120.0, iterations=50, rho=0.9, steps=20, gravity=(0.0, -9.8, 0.0))


def batched_blocks(num_meshes=512, lo=4, hi=24, seed=2024, cell=0.05, jitter=0.25, density=1000.0):
    """The batched configuration: num_meshes jittered grid blocks with dims drawn uniformly from the
    integers [lo, hi]^3 (6 tets per cell), E log-uniform in [1e4, 1e6] Pa, nu uniform in [0.2, 0.45],
    one random face pinned per mesh."""
    rng = np.random.default_rng(seed)
    faces = ("x0", "x1", "y0", "y1", "z0", "z1")
    meshes = []
    for k in range(num_meshes):
        lx, ly, lz = (int(v) for v in rng.integers(lo, hi + 1, size=3))
        E = float(10.0 ** rng.uniform(4.0, 6.0))
        nu = float(rng.uniform(0.2, 0.45))
        face = faces[int(rng.integers(0, 6))]
        meshes.append(jittered_block(lx, ly, lz, cell=cell, jitter=jitter, E=E, nu=nu, density=density,
                                     seed=seed * 1000 + k, pin_face=face))
    return meshes


@dataclass
class Batch:
    """Concatenation of meshes (mesh-local tet ids kept; vertex / tet offsets per mesh)."""

    meshes: list
    vert_offsets: np.ndarray
    tet_offsets: np.ndarray
    rest: np.ndarray
    x: np.ndarray
    v: np.ndarray
    tets_local: np.ndarray
    fixed: np.ndarray
    mu: np.ndarray
    lam: np.ndarray

    @property
    def num_verts(self):
        return int(self.vert_offsets[-1])

    @property
    def num_tets(self):
        return int(self.tet_offsets[-1])

    def split(self, arr):
        """Per-mesh slices of a (num_verts, ...) array."""
        return [arr[self.vert_offsets[m]:self.vert_offsets[m + 1]] for m in range(len(self.meshes))]


def concat(meshes) -> Batch:
    vo = np.zeros(len(meshes) + 1, np.int32)
    to = np.zeros(len(meshes) + 1, np.int32)
    vo[1:] = np.cumsum([m.num_verts for m in meshes])
    to[1:] = np.cumsum([m.num_tets for m in meshes])
    cat = lambda name: np.concatenate([getattr(m, name) for m in meshes])  # noqa: E731
    return Batch(meshes, vo, to, cat("rest"), cat("x"), cat("v"), cat("tets"), cat("fixed"), cat("mu"), cat("lam"))


def diff_beam(seed=33, sigma=0.2):
    """The differentiated configuration: 32x8x8-cell beam (cell 0.05 m, x = 0 face pinned) with per-tet
    log mu, log lambda ~ N(log of the E = 1e5, nu = 0.3 values, sigma); the loss vertices are the 5x5
    subset (j, k in {0, 2, 4, 6, 8}) of the x = max face, with targets = rest position + N(0, 0.01 m).
    Returns (mesh, tip vertex ids, targets (25, 3) float64)."""
    m = beam(32, 8, 8, cell=0.05)
    rng = np.random.default_rng(seed)
    mu0, lam0 = lame(1e5, 0.3)
    m.mu = np.exp(rng.normal(np.log(mu0), sigma, m.num_tets)).astype(np.float32)
    m.lam = np.exp(rng.normal(np.log(lam0), sigma, m.num_tets)).astype(np.float32)
    ijk = m.ijk
    tip = np.flatnonzero((ijk[:, 0] == 32) & (ijk[:, 1] % 2 == 0) & (ijk[:, 2] % 2 == 0))
    target = m.rest[tip].astype(np.float64) + rng.normal(0.0, 0.01, (len(tip), 3))
    m.meta.update(kind="diff_beam", seed=seed, sigma=sigma)
    return m, tip, target


DIFF_SETTINGS = dict(dt=1.0 / 60.0, iterations=30, rho=0.95, steps=30, gravity=(0.0, -9.8, 0.0), checkpoint=10,
                     adjoint_iterations=50, adjoint_rho=0.95)
