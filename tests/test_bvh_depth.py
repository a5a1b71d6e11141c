"""The BVH depth bound: traversal keeps at most one stack entry per level, in
a 64-entry stack like the reference's BvhStack
(src/geometry/accelerators/bvh_stack.h:26), so both BVH builders refuse a
tree whose leaves lie deeper than 64, and no kernel ever sees one.

The degenerate mesh is a row of tiny triangles at x = 2^-k: every binned SAH
split peels a few of the largest off, so the tree's depth grows with the
triangle count (200 triangles: depth 65 in double precision)."""

import ctypes

import numpy as np
import pytest

from math_b200 import painter as P


def geometric_row(count: int, base: float = 2.0):
    v, f = [], []
    for k in range(count):
        x = base ** -k
        s = x * 1e-3
        v += [[x, 0.0, 0.0], [x + s, 0.0, 0.0], [x, s, 0.0]]
        f.append([3 * k, 3 * k + 1, 3 * k + 2])
    return np.array(v, np.float64), np.array(f, np.int32)


def host_build(v, f, n=3, precision=1):
    v = np.ascontiguousarray(v, np.float64)
    f = np.ascontiguousarray(f, np.int32)
    nodes = ctypes.c_longlong(-1)
    depth = ctypes.c_int(-1)
    r = P.lib().nbpt_test_bvh_build(n, precision, P._p(v, P._D), len(v), P._p(f, P._I), len(f),
                                     ctypes.byref(nodes), ctypes.byref(depth))
    return r, nodes.value, depth.value


def test_ordinary_mesh_depth_is_reported():
    from math_b200 import scenes

    p, f = scenes.convex_hull_mesh(scenes.sphere_points(4, 3000, 7))
    r, nodes, depth = host_build(p, f, n=4, precision=0)
    assert r == 0
    assert nodes >= 1 and 1 <= depth <= 64


def test_degenerate_mesh_within_the_bound_builds():
    v, f = geometric_row(100)
    r, nodes, depth = host_build(v, f)
    assert r == 0, P.lib().nbpt_last_error()
    assert 30 <= depth <= 64


def test_degenerate_mesh_beyond_the_bound_is_refused():
    v, f = geometric_row(200)
    r, _, _ = host_build(v, f)
    assert r == -1  # NBPT_ERROR
    msg = P.lib().nbpt_last_error()
    assert b"BVH depth 65 exceeds the traversal stack of 64" in msg


def test_bad_facet_index_is_an_argument_error():
    v, f = geometric_row(4)
    f[0, 0] = 99
    r, _, _ = host_build(v, f)
    assert r == -1
    assert b"out of range" in P.lib().nbpt_last_error()


def degenerate_scene(count: int):
    """The 3-space box with the row of triangles as its mesh, given as mesh
    data in double precision (a float copy of 2^-199 would underflow)."""
    from math_b200 import scenes

    desc = scenes.cornell_3d(size=(8, 8), subdivisions=1)
    desc["shapes"] = [s for s in desc["shapes"] if s["type"] != "mesh"] + [{"type": "mesh", "objects": []}]
    v, f = geometric_row(count)
    v = v * 0.3
    data = [{"vertices": v, "normals": None, "facets": f, "facet_material": np.zeros(len(f), np.int32),
             "material_params": np.array([[0.0, 0.5, 1.0]]), "material_colors": np.array([[0.5, 0.5, 0.5]], np.float32)}]
    return desc, data


@pytest.mark.gpu
@pytest.mark.parametrize("builder", ["device", "host"])
def test_scene_with_a_too_deep_bvh_is_refused(painter, builder):
    desc, data = degenerate_scene(200)
    with pytest.raises(painter.PainterError, match="exceeds the traversal stack of 64"):
        painter.Scene(desc, "double", False, mesh_data=data, bvh_builder=builder)


@pytest.mark.gpu
@pytest.mark.parametrize("builder", ["device", "host"])
def test_deep_bvh_within_the_bound_renders_without_overflow(painter, builder):
    desc, data = degenerate_scene(100)
    s = painter.Scene(desc, "double", False, mesh_data=data, bvh_builder=builder)
    p = s.painter(4, 5, seed=1)
    p.run(1)
    st = p.statistics()
    assert st["stack_overflows"] == 0
    assert st["nonfinite_samples"] == 0
    p.close()
    s.close()
