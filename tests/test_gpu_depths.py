"""Subpath depth bounds: every per-path colour of a seeded double-precision
pass equals the reference painter's for maximum depths 1, 2, 3 and 8, in 3-,
4- (64-bin spectrum) and 5-space.  The walks stop at the depth bound
(bpt.cpp:205-211), connections are cut at s + t - 2 <= max_depth
(connect.cpp:338-342), and the last bounce traces no further ray; the scenes
are the Cornell boxes without their meshes (walls, the parallelotope and the
light), so every colour is compared bit for bit."""

import numpy as np
import pytest

from math_b200 import scenes

pytestmark = pytest.mark.gpu

SCENES = {
    3: (lambda: scenes.cornell_3d(size=(12, 12), subdivisions=1), False, 16),
    4: (lambda: scenes.cornell_4d(size=(5, 5, 5), points=40), True, 8),
    5: (lambda: scenes.cornell_5d(size=(3, 3, 3, 3), points=40), False, 16),
}


def without_meshes(desc):
    desc["shapes"] = [s for s in desc["shapes"] if s["type"] != "mesh"]
    return desc


@pytest.mark.parametrize("n", [3, 4, 5])
@pytest.mark.parametrize("depth", [1, 2, 3, 8])
def test_depth_bound_paths_bit_exact(painter, oracle_lib, n, depth):
    make, spectrum, spp = SCENES[n]
    desc = without_meshes(make())
    o = oracle_lib.Scene(desc, "double", spectrum)
    s = painter.Scene(desc, "double", spectrum)
    p = s.painter(spp, depth, seed=11)
    p.run(1)
    _, colors, valid = p.samples()
    _, ref_colors, ref_valid = o.render_samples(spp, depth, seed=11)
    assert np.array_equal(valid, ref_valid)
    assert np.array_equal(colors, ref_colors)


@pytest.mark.parametrize("n", [3, 4, 5])
def test_pt_paths_bit_exact(painter, oracle_lib, n):
    make, spectrum, spp = SCENES[n]
    desc = without_meshes(make())
    o = oracle_lib.Scene(desc, "double", spectrum)
    o.set_integrator("pt")
    s = painter.Scene(desc, "double", spectrum)
    p = s.painter(spp, 0, seed=11, integrator="pt")
    p.run(1)
    _, colors, valid = p.samples()
    _, ref_colors, ref_valid = o.render_samples(spp, 0, seed=11)
    assert np.array_equal(valid, ref_valid)
    assert np.array_equal(colors, ref_colors)
