"""TetGen input (vbd_tetmesh_b200.tetgen and include/vbd/TetGenIO.h) against the reference driver's
own loader (main.cpp:14-168): its results on the committed samples (tests/golden/tetgen_ref.npz,
from tests/golden/make_tetgen_golden.py) and, where the reference tree is present, live."""
import os
import subprocess

import numpy as np
import pytest

from vbd_tetmesh_b200 import VBDError, mesh_mass, meshgen, surface, tetgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD_DIR = os.path.join(ROOT, "tests", "golden", "tetgen")
GOLD = os.path.join(ROOT, "tests", "golden", "tetgen_ref.npz")
CPP_DIR = os.path.join(ROOT, "tests", "cpp")
CPP_BIN = os.path.join(CPP_DIR, "test_tetgen")
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "ref_tetgen")
DENSITY, MU, LAM = 7800.0e-12, 76923.08, 115384.6
CASES = {"block1": ("block1.node", "block1_cur.node", "block1.ele"), "block0": ("block0.node", None, "block0.ele")}


def read_dump(path):
    raw = open(path, "rb").read()
    n, t = (int(v) for v in np.frombuffer(raw[:8], np.int32))
    o = 8
    rest = np.frombuffer(raw[o:o + 12 * n], np.float32).reshape(n, 3)
    o += 12 * n
    cur = np.frombuffer(raw[o:o + 12 * n], np.float32).reshape(n, 3)
    o += 12 * n
    tets = np.frombuffer(raw[o:o + 16 * t], np.int32).reshape(t, 4)
    o += 16 * t
    fixed = np.frombuffer(raw[o:o + n], np.uint8)
    o += n
    mass = np.frombuffer(raw[o:o + 4 * n], np.float32)
    return dict(rest=rest, current=cur, tets=tets, fixed=fixed, mass=mass)


def run_binary(binary, rest, cur, ele, out):
    obj = str(out) + ".obj"
    args = [binary, rest, cur or "", ele, repr(DENSITY), repr(MU), repr(LAM), str(out), obj]
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    res = read_dump(out)
    res["obj"] = open(obj).read()
    return res


def python_load(rest, cur, ele):
    m = tetgen.load_tetgen(rest, ele, cur, density=DENSITY, mu=MU, lam=LAM)
    mass, _ = mesh_mass(m.rest, m.tets, m.density)
    return dict(rest=m.rest, current=m.x, tets=m.tets, fixed=m.fixed, mass=mass, obj=surface.obj_text(m.x, m.tets))


def assert_same(a, b):
    for k in ("rest", "current", "tets", "fixed", "mass"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    assert a["obj"] == b["obj"], "OBJ text differs"


def paths(case):
    rest, cur, ele = CASES[case]
    return os.path.join(GOLD_DIR, rest), (os.path.join(GOLD_DIR, cur) if cur else None), os.path.join(GOLD_DIR, ele)


@pytest.mark.parametrize("case", list(CASES))
def test_python_loader_matches_reference_loader_golden(case):
    gold = np.load(GOLD)
    ref = {k: gold[f"{case}/{k}"] for k in ("rest", "current", "tets", "fixed", "mass")}
    ref["obj"] = str(gold[f"{case}/obj"])
    ours = python_load(*paths(case))
    assert_same(ours, ref)
    assert ref["fixed"].sum() > 0


@pytest.mark.parametrize("case", list(CASES))
def test_cpp_loader_matches_reference_loader_golden(case, tmp_path):
    if not os.path.exists(CPP_BIN):
        subprocess.run(["make", "-C", CPP_DIR, "test_tetgen"], check=True, capture_output=True)
    gold = np.load(GOLD)
    ref = {k: gold[f"{case}/{k}"] for k in ("rest", "current", "tets", "fixed", "mass")}
    ref["obj"] = str(gold[f"{case}/obj"])
    rest, cur, ele = paths(case)
    assert_same(run_binary(CPP_BIN, rest, cur, ele, tmp_path / "ours.bin"), ref)


@pytest.mark.skipif(not os.path.exists(REF_BIN), reason="reference loader not built (make -C oracle reftetgen)")
@pytest.mark.parametrize("seed,base,fmt", [(1, 1, "%.6f"), (2, 0, "%.9e"), (3, 1, "%.3f")])
def test_loaders_match_reference_loader_live(seed, base, fmt, tmp_path):
    pos, tets, _ = meshgen.grid(4, 5, 3, cell=0.7, jitter=0.25, seed=seed)
    cur = pos * np.array([1.0, 0.97, 1.01])

    def node(path, p):
        with open(path, "w") as f:
            f.write(f"{len(p)}  3  0  0\n")
            for i, q in enumerate(p):
                f.write(f"{i + base}  " + "  ".join(fmt % v for v in q) + "\n")

    node(tmp_path / "r.node", pos)
    node(tmp_path / "c.node", cur)
    with open(tmp_path / "m.ele", "w") as f:
        f.write(f"{len(tets)}  4  0\n")
        for t, q in enumerate(tets):
            f.write(f"{t + base}  " + "  ".join(str(int(v) + base) for v in q) + "\n")
    args = (str(tmp_path / "r.node"), str(tmp_path / "c.node"), str(tmp_path / "m.ele"))
    ref = run_binary(REF_BIN, *args, tmp_path / "ref.bin")
    if not os.path.exists(CPP_BIN):
        subprocess.run(["make", "-C", CPP_DIR, "test_tetgen"], check=True, capture_output=True)
    assert_same(run_binary(CPP_BIN, *args, tmp_path / "ours.bin"), ref)
    assert_same(python_load(*args), ref)


def test_attribute_columns_and_comments_round_trip(tmp_path):
    """TetGen files with attribute / boundary-marker columns and comment lines are read by their
    format; main.cpp's loader would take the extra columns as the next record's fields."""
    m = meshgen.jittered_block(4, 3, 3, seed=5)
    for base in (0, 1):
        node, ele = tetgen.write_tetgen(str(tmp_path / f"b{base}"), m.rest, m.tets, index_base=base)
        # add a boundary-marker column and a comment line in the middle of the file
        lines = open(node).read().splitlines()
        lines = [lines[0]] + ["# node records"] + [ln + "  1" for ln in lines[1:-1]] + [lines[-1]]
        open(node, "w").write("\n".join(lines) + "\n")
        got = tetgen.load_tetgen(node, ele, None, mu=1.0, lam=1.0, pin_axes=())
        np.testing.assert_array_equal(got.rest, m.rest)
        np.testing.assert_array_equal(got.tets, m.tets)
        assert got.fixed.sum() == 0


def test_pinning_rule():
    rng = np.random.default_rng(3)
    x = rng.uniform(-3, 7, (500, 3)).astype(np.float32)
    for axis in range(3):
        lo, hi = x[:, axis].min(), x[:, axis].max()
        thr = np.float32(lo + (hi - lo) * np.float32(0.05))
        expect = (x[:, axis] <= thr).astype(np.uint8)
        np.testing.assert_array_equal(tetgen.pin_low_fraction(x, axis, 0.05), expect)


def test_loader_errors(tmp_path):
    with pytest.raises(VBDError):
        tetgen.read_node(str(tmp_path / "missing.node"))
    m = meshgen.jittered_block(2, 2, 2, seed=1)
    node, ele = tetgen.write_tetgen(str(tmp_path / "m"), m.rest, m.tets, index_base=1)
    with pytest.raises(VBDError):
        tetgen.read_ele(ele, 1, num_nodes=5)  # ids beyond the node count
    short = tmp_path / "short.node"
    tetgen.write_tetgen(str(tmp_path / "short"), m.rest[:-1], m.tets[:1], index_base=1)
    with pytest.raises(VBDError):
        tetgen.load_tetgen(node, ele, str(short))  # rest / current count mismatch
    # missing current-shape file: the rest positions are used (main.cpp:66-71)
    got = tetgen.load_tetgen(node, ele, str(tmp_path / "absent.node"), mu=1.0, lam=1.0)
    np.testing.assert_array_equal(got.x, got.rest)


def test_main_cpp_material_in_float32():
    mu, lam = tetgen.lame_f32(200.0e3, 0.3)
    assert mu == float(np.float32(200.0e3) / (np.float32(2.0) * (np.float32(1.0) + np.float32(0.3))))
    assert abs(mu - 76923.08) < 0.01 and abs(lam - 115384.6) < 0.1


def test_surface_faces_of_a_grid():
    m = meshgen.jittered_block(3, 4, 5, seed=2)
    faces = surface.extract_surface_faces(m.tets)
    assert len(faces) == 2 * 2 * (3 * 4 + 4 * 5 + 3 * 5)
    # each boundary triangle is a face of exactly one tet, in the orientation that tet lists it
    listed = {tuple(t[list(f)]) for t in m.tets for f in surface.FACE_ORDER}
    assert all(tuple(f) in listed for f in faces)
    keys = np.sort(faces, axis=1)
    assert len({tuple(k) for k in keys}) == len(faces)
