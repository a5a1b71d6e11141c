"""Scenes with meshes read from n-dimensional OBJ and STL files, rendered by
the GPU painter and by the reference painter (its own loaders, compiled into
the oracle) from the same files: the facet records, the BVH and every
per-path colour of a seeded double-precision pass are equal.  The files cover
normals given per corner (OBJ "vn"), flat facets (STL, OBJ without "vn"),
materials with Kd colours, relative indices and comments, in 3-, 4- and
5-space."""

import numpy as np
import pytest

from math_b200 import scenes
from mesh_file_writers import obj_extension, stl_extension, write_obj, write_stl_ascii, write_stl_binary

pytestmark = pytest.mark.gpu


def scene_with_file(n, path, size):
    if n == 3:
        desc = scenes.cornell_3d(size=size, subdivisions=1)
        matrix = scenes.transform_matrix(n, 0.4, [0.0, -0.6, 0.1])
    elif n == 4:
        desc = scenes.cornell_4d(size=size, points=40)
        matrix = scenes.transform_matrix(n, 0.4, [-0.35, -0.55, -0.25, 0.15])
    else:
        desc = scenes.cornell_5d(size=size, points=40)
        matrix = scenes.transform_matrix(n, 0.4, [0.0, -0.5, 0.0, 0.0, 0.0])
    mesh = [s for s in desc["shapes"] if s["type"] == "mesh"][0]
    mesh["objects"] = [{"file": str(path), "matrix": np.asarray(matrix).tolist(), "metalness": 0.1,
                        "roughness": 0.3, "color": [0.6, 0.7, 0.8], "alpha": 1.0}]
    return desc


def mesh(n):
    if n == 3:
        p, f = scenes.icosphere(3)
    else:
        p, f = scenes.convex_hull_mesh(scenes.sphere_points(n, 600 if n == 4 else 200, 5))
    return np.asarray(p, np.float32), np.asarray(f)


def write(kind, tmp_path, n):
    p, f = mesh(n)
    if kind == "obj_normals":
        path = tmp_path / ("m" + obj_extension(n))
        write_obj(path, p, f, normals=p / np.linalg.norm(p, axis=1, keepdims=True),
                  materials={"warm": (0.9, 0.5, 0.2), "cold": (0.2, 0.4, 0.9)},
                  facet_material=[("warm", "cold", None)[i % 3] for i in range(len(f))], relative_every=4)
    elif kind == "obj_mixed":
        path = tmp_path / ("m" + obj_extension(n))
        write_obj(path, p, f, normals=p / np.linalg.norm(p, axis=1, keepdims=True),
                  with_normals=np.arange(len(f)) % 2 == 0)
    elif kind == "stl_ascii":
        path = tmp_path / ("m" + stl_extension(n))
        write_stl_ascii(path, p, f)
    else:
        path = tmp_path / ("m" + stl_extension(n))
        write_stl_binary(path, p, f)
    return path


CASES = [(3, "obj_normals"), (3, "obj_mixed"), (3, "stl_binary"), (4, "obj_normals"), (4, "stl_ascii"),
         (5, "obj_mixed"), (5, "stl_binary")]


@pytest.mark.parametrize("n,kind", CASES)
def test_file_scene_matches_reference(painter, oracle_lib, tmp_path, n, kind):
    path = write(kind, tmp_path, n)
    size = {3: (12, 12), 4: (5, 5, 5), 5: (3, 3, 3, 3)}[n]
    desc = scene_with_file(n, path, size)
    o = oracle_lib.Scene(desc, "double", False)
    s = painter.Scene(desc, "double", False)
    ref = o.mesh_dump()
    mine = s.mesh_export(0)
    assert np.array_equal(mine["planes"], ref["planes"])
    assert np.array_equal(mine["node_info"], ref["node_info"])
    assert np.array_equal(mine["node_lo"], ref["node_bounds"][:, 0])
    assert np.array_equal(mine["node_hi"], ref["node_bounds"][:, 1])
    assert np.array_equal(mine["indices"], ref["indices"])
    p = s.painter(8, 5, seed=4)
    p.run(1)
    _, colors, valid = p.samples()
    _, ref_colors, ref_valid = o.render_samples(8, 5, seed=4)
    assert np.array_equal(valid, ref_valid)
    assert np.array_equal(colors, ref_colors)
