"""Mesh files (n-dimensional OBJ and STL) without a GPU: the library's loader
accepts and rejects the same files as the reference's loaders
(src/model/mesh/file/load_obj.cpp, load_stl.cpp, compiled into the oracle),
reads the same arrays from them (tests/mesh_file_check.cpp against
oracle_mesh_file_arrays, on files large enough for the loader's host
threads), and names file dimensions as file_type.cpp does."""

import numpy as np
import pytest

from math_b200 import scenes
from mesh_file_writers import obj_extension, stl_extension, write_obj, write_stl_ascii, write_stl_binary


def lib():
    from math_b200 import painter

    try:
        return painter, painter.lib()
    except painter.PainterError as e:
        pytest.skip(str(e))


def tetra(n):
    p, f = scenes.icosphere(1) if n == 3 else scenes.convex_hull_mesh(scenes.sphere_points(n, 40, 1))
    return np.asarray(p, np.float32), np.asarray(f)


def add_file(L, n, path):
    from math_b200 import painter as P

    h = L.nbpt_scene_create(n, 0, 0)
    m = np.eye(n + 1).reshape(-1)
    rgb = np.array([0.5, 0.5, 0.5], np.float32)
    r = L.nbpt_scene_add_mesh_file(h, str(path).encode(), P._p(m, P._D), 0.0, 0.3, P._p(rgb, P._F), 1.0)
    err = L.nbpt_last_error().decode() if r < 0 else ""
    L.nbpt_scene_destroy(h)
    return r, err


def oracle_add_file(oracle_lib, n, path):
    desc = scenes.cornell_3d(size=(4, 4), subdivisions=1) if n == 3 else scenes.cornell_4d(size=(2, 2, 2), points=40)
    if n == 5:
        desc = scenes.cornell_5d(size=(2, 2, 2, 2), points=40)
    mesh = [s for s in desc["shapes"] if s["type"] == "mesh"][0]
    mesh["objects"] = [{"file": str(path), "matrix": np.eye(n + 1).tolist(), "metalness": 0.0,
                        "roughness": 0.3, "color": [0.5, 0.5, 0.5], "alpha": 1.0}]
    try:
        oracle_lib.Scene(desc, "double", False)
        return 0
    except Exception:
        return -1


def test_file_dimension():
    P, L = lib()
    for name, n in (("a.obj", 3), ("a.stl", 3), ("b.obj4", 4), ("b.STL5", 5), ("c.obj3", 3)):
        assert L.nbpt_mesh_file_dimension(name.encode()) == n
    assert L.nbpt_mesh_file_dimension(b"a.txt") < 0


@pytest.mark.parametrize("n", [3, 4, 5])
def test_well_formed_files_load(tmp_path, n, oracle_lib):
    P, L = lib()
    p, f = tetra(n)
    files = [tmp_path / ("a" + obj_extension(n)), tmp_path / ("b" + stl_extension(n)),
             tmp_path / ("c" + stl_extension(n))]
    write_obj(files[0], p, f, normals=p / np.linalg.norm(p, axis=1, keepdims=True),
              with_normals=np.arange(len(f)) % 2 == 0, materials={"red": (0.8, 0.1, 0.1)},
              facet_material=["red" if i % 3 == 0 else None for i in range(len(f))], relative_every=5)
    write_stl_ascii(files[1], p, f)
    write_stl_binary(files[2], p, f)
    for path in files:
        r, err = add_file(L, n, path)
        assert r >= 0, err
        assert oracle_add_file(oracle_lib, n, path) == 0


MALFORMED_OBJ = {
    "zero index": "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 0 1 2\n",
    "too few corners": "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2\n",
    "index out of range": "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4\n",
    "mixed normals": "v 0 0 0\nv 1 0 0\nv 0 1 0\nvn 0 0 1\nf 1//1 2 3\n",
    "short vertex": "v 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n",
    "bad separator": "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1x 2 3\n",
    "no facets": "v 0 0 0\n",
    "unknown material": "v 0 0 0\nv 1 0 0\nv 0 1 0\nusemtl m\nf 1 2 3\n",
    "degenerate only": "v 0 0 0\nv 1 0 0\nv 2 0 0\nf 1 2 3\n",
    "too many corners": "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3 1 2 3 1 2\n",
}


@pytest.mark.parametrize("case", list(MALFORMED_OBJ))
def test_malformed_obj_rejected_like_the_reference(tmp_path, case, oracle_lib):
    P, L = lib()
    path = tmp_path / "m.obj"
    path.write_text(MALFORMED_OBJ[case])
    r, err = add_file(L, 3, path)
    assert r < 0 and err
    assert oracle_add_file(oracle_lib, 3, path) < 0


MALFORMED_STL = {
    "no solid": "facet normal 0 0 1\n",
    "no endsolid": "solid x\n facet normal 0 0 1\n  outer loop\n   vertex 0 0 0\n   vertex 1 0 0\n"
                   "   vertex 0 1 0\n  endloop\n endfacet\n",
    "short vertex": "solid x\n facet normal 0 0 1\n  outer loop\n   vertex 0 0\n   vertex 1 0 0\n"
                    "   vertex 0 1 0\n  endloop\n endfacet\nendsolid x\n",
    "text after end": "solid x\n facet normal 0 0 1\n  outer loop\n   vertex 0 0 0\n   vertex 1 0 0\n"
                      "   vertex 0 1 0\n  endloop\n endfacet\nendsolid x\nmore\n",
}


@pytest.mark.parametrize("case", list(MALFORMED_STL))
def test_malformed_stl_rejected_like_the_reference(tmp_path, case, oracle_lib):
    P, L = lib()
    path = tmp_path / "m.stl"
    path.write_text(MALFORMED_STL[case])
    r, err = add_file(L, 3, path)
    assert r < 0 and err
    assert oracle_add_file(oracle_lib, 3, path) < 0


def test_dimension_mismatch(tmp_path):
    P, L = lib()
    path = tmp_path / "a.obj4"
    path.write_text("v 0 0 0 0\n")
    r, err = add_file(L, 3, path)
    assert r < 0 and "dimension" in err


# --------------------------------------------------------------------------
# what the loader reads, array for array against the reference's loaders


def build_check(tmp_path):
    """tests/mesh_file_check.cpp with the library's loader, compiled here."""
    import shutil
    import subprocess
    from pathlib import Path

    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    here = Path(__file__).resolve().parent
    csrc = here.parent / "math_b200" / "csrc"
    exe = tmp_path / "mesh_file_check"
    subprocess.run(["g++", "-std=c++20", "-O2", "-ffp-contract=off", f"-I{csrc}", str(here / "mesh_file_check.cpp"),
                    str(csrc / "mesh_files.cpp"), "-pthread", "-o", str(exe)], check=True)
    return exe


def read_check(exe, path, n, out):
    import subprocess

    subprocess.run([str(exe), str(path), str(n), str(out)], check=True)
    data = out.read_bytes()
    v, m, f = np.frombuffer(data[:24], np.int64)
    o = 24
    arrays = {}
    for name, dtype, shape in (("vertices", np.float32, (v, n)), ("normals", np.float32, (m, n)),
                               ("facet_vertices", np.int32, (f, n)), ("facet_normals", np.int32, (f, n)),
                               ("has_normal", np.uint8, (f,)), ("facet_material", np.int32, (f,))):
        size = int(np.prod(shape)) * np.dtype(dtype).itemsize
        arrays[name] = np.frombuffer(data[o:o + size], dtype).reshape(shape)
        o += size
    assert o == len(data)
    return arrays


def big_mesh(n):
    """Meshes large enough that the loader splits the work over host threads
    (more than 65,536 STL corners, more than 8,192 OBJ lines)."""
    if n == 3:
        p, f = scenes.icosphere(6)
    else:
        p, f = scenes.convex_hull_mesh(scenes.sphere_points(n, 5000 if n == 4 else 1500, 6))
    p = np.asarray(p, np.float32)
    # signed zeros, which the loaders merge, in some coordinates
    p[::5, 0] = 0.0
    p[2::5, 0] = -0.0
    return p, np.asarray(f)


@pytest.mark.parametrize("n", [3, 4, 5])
def test_loaded_arrays_match_the_reference(tmp_path, n, oracle_lib):
    """Vertices (merged STL corners numbered by first appearance), normals,
    facet indices, flags and materials equal the reference loaders' output
    bit for bit, for OBJ with normals on some facets, materials and relative
    indices, and for ASCII and binary STL, one of them with NaN corners."""
    import struct

    from mesh_file_writers import facet_normals

    exe = build_check(tmp_path)
    p, f = big_mesh(n)
    nrm = p / np.maximum(np.linalg.norm(p, axis=1, keepdims=True), 1e-30)
    files = {"obj": tmp_path / ("m" + obj_extension(n)), "ascii": tmp_path / ("a" + stl_extension(n)),
             "binary": tmp_path / ("b" + stl_extension(n)), "nan": tmp_path / ("c" + stl_extension(n))}
    write_obj(files["obj"], p, f, normals=nrm, with_normals=(np.arange(len(f)) // 40) % 3 != 0,
              materials={"red": (0.8, 0.1, 0.1), "blue": (0.1, 0.1, 0.8)},
              facet_material=[("red", None, "blue")[(i // 70) % 3] for i in range(len(f))], relative_every=3)
    write_stl_ascii(files["ascii"], p, f)
    write_stl_binary(files["binary"], p, f)
    q = p.copy()
    q[7, 1] = np.nan
    q[11, 0] = np.nan
    fn = facet_normals(p.astype(np.float64), f).astype(np.float32)
    with open(files["nan"], "wb") as h:
        h.write(b"binary STL with NaN corners".ljust(80, b" "))
        h.write(struct.pack("<I", len(f)))
        for facet, normal in zip(f, fn):
            h.write(normal.tobytes())
            h.write(q[facet].tobytes())
    for kind, path in files.items():
        mine = read_check(exe, path, n, tmp_path / f"{kind}.bin")
        ref = oracle_lib.mesh_file_arrays(path, n)
        for name in ("vertices", "normals"):
            assert mine[name].tobytes() == ref[name].tobytes(), (kind, name)
        for name in ("facet_vertices", "facet_normals", "has_normal", "facet_material"):
            assert np.array_equal(mine[name], ref[name]), (kind, name)
        if kind != "obj":
            # STL corners merged: fewer vertices than corners
            assert len(mine["vertices"]) < len(f) * n
