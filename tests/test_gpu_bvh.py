"""The mesh BVH built on the GPU against the host build, record for record.

The host builder follows the reference's sequential build step for step
(its trees equal the reference's: test_gpu_parity.py checks both against the
compiled reference's fixtures), so equal node bounds, node records and leaf
index slots show the GPU builder reproduces the reference's tree: the same
SAH decisions, the same std::partition element order, the same depth-first
layout.  Small meshes exercise the one-warp subtree build, large ones the
per-level kernels.
"""

import numpy as np
import pytest

from math_b200 import scenes

pytestmark = pytest.mark.gpu

CASES = {
    "cornell3d_small": (lambda: scenes.cornell_3d(size=(8, 8), subdivisions=1), False),
    "cornell3d": (lambda: scenes.cornell_3d(size=(8, 8), subdivisions=5), False),
    "cornell3d_fine": (lambda: scenes.cornell_3d(size=(8, 8), subdivisions=7), False),
    "cornell4d": (lambda: scenes.cornell_4d(size=(4, 4, 4), points=20000), True),
    "cornell5d": (lambda: scenes.cornell_5d(size=(3, 3, 3, 3), points=2000), False),
    "sphere4d": (lambda: scenes.sphere_4d(size=(4, 4, 4), points=30000, buckets=8), False),
}


def export_both(painter, desc, precision, spectrum):
    out = []
    for builder in ("device", "host"):
        s = painter.Scene(desc, precision, spectrum, bvh_builder=builder)
        out.append(s.mesh_export(0))
        s.close()
    return out


@pytest.mark.parametrize("precision", ["float", "double"])
@pytest.mark.parametrize("name", list(CASES))
def test_device_bvh_equals_host_bvh(painter, name, precision):
    make, spectrum = CASES[name]
    device, host = export_both(painter, make(), precision, spectrum)
    assert len(device["node_info"]) == len(host["node_info"])
    assert np.array_equal(device["node_info"], host["node_info"])
    assert np.array_equal(device["node_lo"], host["node_lo"])
    assert np.array_equal(device["node_hi"], host["node_hi"])
    assert np.array_equal(device["indices"], host["indices"])
    assert np.array_equal(device["planes"], host["planes"])


def test_device_bvh_renders_as_host_bvh(painter):
    """Same tree, same paths: per-sample colours of one pass are equal."""
    desc = scenes.cornell_4d(size=(6, 6, 6), points=2000)
    colors = []
    for builder in ("device", "host"):
        s = painter.Scene(desc, "double", True, bvh_builder=builder)
        p = s.painter(8, 6, seed=3)
        p.run(1)
        colors.append(p.samples()[1])
        p.close()
        s.close()
    assert np.array_equal(colors[0], colors[1])


def test_bvh_builder_errors(painter):
    desc = scenes.cornell_3d(size=(4, 4), subdivisions=1)
    with pytest.raises(KeyError):
        painter.Scene(desc, "float", False, bvh_builder="cpu")
    L = painter.lib()
    h = L.nbpt_scene_create(3, 0, 0)
    assert L.nbpt_scene_set_bvh_builder(h, 2) < 0
    assert "BVH builder" in L.nbpt_last_error().decode()
    L.nbpt_scene_destroy(h)
