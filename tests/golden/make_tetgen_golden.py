"""Writes the TetGen sample meshes under tests/golden/tetgen/ and, with the reference driver's own
loader (oracle/_ref/ref_tetgen, built by `make -C oracle reftetgen` where the reference sources
are present), records what it loads from them, and the OBJ file TetMesh::exportToObj writes for them, in
tests/golden/tetgen_ref.npz.

Samples (seeded, decimal text as TetGen writes it, "%.6f"; no attribute or boundary-marker
columns, the only records main.cpp's loader reads correctly -- its stream keeps unread tokens, so
an extra column is taken as the next record's index):
  block1: 1-based ids, trailing '#' comments, and a current-shape file block1_cur.node (y
          compressed by 2%, seeded noise);
  block0: 0-based ids, no current-shape file.
Run:  python tests/golden/make_tetgen_golden.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from vbd_tetmesh_b200 import meshgen  # noqa: E402

OUT_DIR = os.path.join(HERE, "tetgen")
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_tetgen")
MATERIAL = (7800.0e-12, 76923.08, 115384.6)  # density, mu, lambda as main.cpp's E = 200e3, nu = 0.3
CASES = {"block1": ("block1.node", "block1_cur.node", "block1.ele"), "block0": ("block0.node", "", "block0.ele")}


def write_samples():
    os.makedirs(OUT_DIR, exist_ok=True)
    pos, tets, _ = meshgen.grid(5, 3, 4, cell=2.5, jitter=0.2, seed=17)
    rng = np.random.default_rng(18)
    cur = pos.copy()
    cur[:, 1] *= 0.98
    cur += rng.normal(0.0, 0.01, cur.shape)
    for name, base, with_cur in (("block1", 1, True), ("block0", 0, False)):
        def node_file(path, p):
            with open(path, "w") as f:
                f.write(f"{len(p)}  3  0  0\n")
                for i, q in enumerate(p):
                    f.write(f"    {i + base}    {q[0]:.6f}  {q[1]:.6f}  {q[2]:.6f}\n")
                f.write("# Generated by make_tetgen_golden.py\n")
        node_file(os.path.join(OUT_DIR, f"{name}.node"), pos)
        if with_cur:
            node_file(os.path.join(OUT_DIR, f"{name}_cur.node"), cur)
        with open(os.path.join(OUT_DIR, f"{name}.ele"), "w") as f:
            f.write(f"{len(tets)}  4  0\n")
            for t, q in enumerate(tets):
                f.write(f"    {t + base}    {q[0] + base}  {q[1] + base}  {q[2] + base}  {q[3] + base}\n")
            f.write("# Generated by make_tetgen_golden.py\n")


def read_dump(path):
    raw = open(path, "rb").read()
    n, t = np.frombuffer(raw[:8], np.int32)
    o = 8
    rest = np.frombuffer(raw[o:o + 12 * n], np.float32).reshape(n, 3); o += 12 * n
    cur = np.frombuffer(raw[o:o + 12 * n], np.float32).reshape(n, 3); o += 12 * n
    tets = np.frombuffer(raw[o:o + 16 * t], np.int32).reshape(t, 4); o += 16 * t
    fixed = np.frombuffer(raw[o:o + n], np.uint8); o += n
    mass = np.frombuffer(raw[o:o + 4 * n], np.float32)
    return dict(rest=rest, current=cur, tets=tets, fixed=fixed, mass=mass)


def run_loader(binary, case, out):
    rest, cur, ele = CASES[case]
    d = OUT_DIR
    obj = out + ".obj"
    args = [binary, os.path.join(d, rest), os.path.join(d, cur) if cur else "", os.path.join(d, ele),
            *(repr(v) for v in MATERIAL), out, obj]
    subprocess.run(args, check=True, capture_output=True)
    res = read_dump(out)
    res["obj"] = np.array(open(obj).read())  # TetMesh::exportToObj of the loaded mesh
    return res


def main():
    write_samples()
    if not os.path.exists(HARNESS):
        print("reference loader not built; wrote the samples only")
        return
    data = {}
    with tempfile.TemporaryDirectory() as tmp:
        for case in CASES:
            for k, v in run_loader(HARNESS, case, os.path.join(tmp, f"{case}.bin")).items():
                data[f"{case}/{k}"] = v
    np.savez_compressed(os.path.join(HERE, "tetgen_ref.npz"), **data)
    print("wrote tetgen_ref.npz", {k: v.shape for k, v in data.items()})


if __name__ == "__main__":
    main()
