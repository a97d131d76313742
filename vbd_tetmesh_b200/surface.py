"""Boundary surface of a tet mesh and Wavefront OBJ export, as TetMesh::extractSurfaceFaces and
TetMesh::exportToObj do it (TetMesh.h:80-186): every tet contributes its four faces
(v0 v2 v1), (v0 v1 v3), (v0 v3 v2), (v1 v2 v3); a face met exactly once is on the boundary and keeps
the orientation it had there; boundary faces are listed in the order of their sorted vertex ids.
Positions typically come from a solver readback (``GPUSolver.get_positions``)."""
from __future__ import annotations

import numpy as np

FACE_ORDER = ((0, 2, 1), (0, 1, 3), (0, 3, 2), (1, 2, 3))


def extract_surface_faces(tets) -> np.ndarray:
    """(F, 3) int32 boundary triangles."""
    tets = np.asarray(tets, np.int64).reshape(-1, 4)
    if tets.shape[0] == 0:
        return np.zeros((0, 3), np.int32)
    oriented = np.concatenate([tets[:, list(f)] for f in FACE_ORDER], axis=0)  # face-major
    # order of first occurrence: tet index, then face index within the tet
    first_rank = np.concatenate([np.arange(tets.shape[0]) * 4 + k for k in range(4)])
    keys = np.sort(oriented, axis=1)
    order = np.lexsort((first_rank, keys[:, 2], keys[:, 1], keys[:, 0]))
    k = keys[order]
    new = np.ones(len(k), bool)
    new[1:] = np.any(k[1:] != k[:-1], axis=1)
    starts = np.flatnonzero(new)
    counts = np.diff(np.append(starts, len(k)))
    once = starts[counts == 1]
    return oriented[order[once]].astype(np.int32)


def obj_text(positions, tets) -> str:
    """The text TetMesh::exportToObj writes (C++ stream defaults: 6 significant digits)."""
    pos = np.asarray(positions, np.float32).reshape(-1, 3)
    tets = np.asarray(tets).reshape(-1, 4)
    faces = extract_surface_faces(tets)
    out = [f"# TetMesh OBJ Export\n# Vertices: {len(pos)}\n# Tetrahedra: {len(tets)}\n\n"]
    out.extend(f"v {float(p[0]):g} {float(p[1]):g} {float(p[2]):g}\n" for p in pos)
    out.append("\n")
    out.append(f"# Surface Triangles: {len(faces)}\n")
    out.extend(f"f {f[0] + 1} {f[1] + 1} {f[2] + 1}\n" for f in faces)
    return "".join(out)


def export_obj(path, positions, tets) -> int:
    """Writes the OBJ file; returns the number of boundary triangles."""
    text = obj_text(positions, tets)
    with open(path, "w") as f:
        f.write(text)
    return text.count("\nf ")
