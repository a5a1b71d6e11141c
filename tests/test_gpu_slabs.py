"""The slab painter (nbpt_painter_create_slab), the GPU side of a render split
across ranks by slabs of the screen (math_b200/tiles.py): on one GPU, the
slabs of a 2- and 3-way split rendered one after another and put together
equal the whole-screen render bit for bit, for both integrators and in 3-,
4- (spectral) and 5-space, and a slab's samples are the whole render's
samples of its rows and halo."""

from __future__ import annotations

import numpy as np
import pytest

from math_b200 import painter as P
from math_b200 import scenes, tiles

pytestmark = pytest.mark.gpu

SCENES = {
    "3-space": (lambda: scenes.cornell_3d(size=(20, 17), subdivisions=2), False),
    "4-space spectral": (lambda: scenes.cornell_4d(size=(6, 5, 7), points=400), True),
    "5-space": (lambda: scenes.cornell_5d(size=(4, 3, 4, 5), points=150), False),
}


@pytest.mark.parametrize("name", list(SCENES))
@pytest.mark.parametrize("integrator", ["bpt", "pt"])
@pytest.mark.parametrize("precision", ["double", "float"])
def test_slabs_put_together_equal_the_whole_render(painter, name, integrator, precision):
    make, spectrum = SCENES[name]
    desc = make()
    s = P.Scene(desc, precision, spectrum)
    whole = s.painter(16, 5, seed=2, integrator=integrator)
    whole.run(2)
    ref_rgb, ref_rgba = whole.images()
    rows = s.size[-1]
    for world in (2, 3):
        rgb, rgba, paths = [], [], 0
        for rank in range(world):
            slab = tiles.slab_rows(rows, rank, world)
            p = s.painter(16, 5, seed=2, integrator=integrator, slab=slab)
            p.run(2)
            a, b = p.images()
            rgb.append(a)
            rgba.append(b)
            paths += p.statistics()["sample_count"]
            p.close()
        assert np.array_equal(tiles.assemble(rgb), ref_rgb)
        assert np.array_equal(tiles.assemble(rgba), ref_rgba)
        # the halo rows are rendered twice
        assert paths > s.pixels * whole.spp
    whole.close()
    s.close()


def test_slab_samples_are_the_whole_renders(painter):
    desc = scenes.cornell_3d(size=(16, 12), subdivisions=2)
    s = P.Scene(desc, "double", False)
    whole = s.painter(16, 5, seed=4)
    whole.run(1)
    points, colors, valid = whole.samples()
    p = s.painter(16, 5, seed=4, slab=(5, 9))
    p.run(1)
    sp, sc, sv = p.samples()
    first, last = tiles.pixel_range(s.size, *tiles.source_rows(12, 5, 9))
    assert np.array_equal(sp, points[first:last])
    assert np.array_equal(sc, colors[first:last])
    assert np.array_equal(sv, valid[first:last])
    assert p.statistics()["sample_count"] == (last - first) * p.spp
    with pytest.raises(P.PainterError, match="outside the screen"):
        s.painter(16, 5, seed=4, slab=(9, 13))
    s.close()
