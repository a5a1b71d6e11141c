"""The estimator's per-pixel sums in float or double (nbpt_painter_options'
pixel_sums).

Float sums are the reference's (its Color is float in both instantiations,
src/color/color.h:416-417; merges in src/painter/pixels/pixels.cpp:83-95 and
samples/com/merge.h:199-233) and keep a double-precision render's image the
reference's bit for bit.  Double sums run the same merges, the same
held-out selection and the same order, with the radiance and weight sums in
double; the single-precision trace uses them by default.  From the same
samples the two images therefore differ only by the float rounding of the
sums."""

from __future__ import annotations

import numpy as np
import pytest

from math_b200 import painter as P
from math_b200 import scenes

pytestmark = pytest.mark.gpu

SCENES = {
    "3-space": (lambda: scenes.cornell_3d(size=(24, 20), subdivisions=2), False),
    "4-space spectral": (lambda: scenes.cornell_4d(size=(6, 5, 7), points=400), True),
    "5-space": (lambda: scenes.cornell_5d(size=(4, 3, 4, 5), points=150), False),
}


def render(scene, pixel_sums, passes, spp=16, integrator="bpt"):
    p = scene.painter(spp, 5, seed=3, integrator=integrator, pixel_sums=pixel_sums)
    p.run(passes)
    rgb, rgba = p.images()
    samples = p.samples()
    p.close()
    return rgb, rgba, samples


@pytest.mark.parametrize("name", list(SCENES))
@pytest.mark.parametrize("precision", ["double", "float"])
def test_default_sums_by_precision(name, precision):
    make, spectrum = SCENES[name]
    s = P.Scene(make(), precision, spectrum)
    default = render(s, None, 2)
    same = render(s, "float" if precision == "double" else "double", 2)
    assert np.array_equal(default[0], same[0])
    assert np.array_equal(default[1], same[1])
    s.close()


@pytest.mark.parametrize("name", list(SCENES))
@pytest.mark.parametrize("integrator", ["bpt", "pt"])
def test_double_sums_differ_from_float_by_rounding(name, integrator):
    """Same samples (the path kernels do not depend on the sums), images
    within the float rounding of the sums: relative 1e-5 per channel, and at
    least one pixel differs after several passes in 3- and 5-space (the
    sums of many samples round differently)."""
    make, spectrum = SCENES[name]
    s = P.Scene(make(), "double", spectrum)
    f_rgb, f_rgba, f_samples = render(s, "float", 6, integrator=integrator)
    d_rgb, d_rgba, d_samples = render(s, "double", 6, integrator=integrator)
    for a, b in zip(f_samples, d_samples):
        assert np.array_equal(a, b)
    assert np.isfinite(d_rgb).all() and np.isfinite(d_rgba).all()
    assert np.allclose(d_rgb, f_rgb, rtol=1e-5, atol=1e-7)
    assert np.allclose(d_rgba, f_rgba, rtol=1e-5, atol=1e-7)
    # pixels with samples and pixels without them are the same in both
    assert np.array_equal(d_rgba[:, 3] > 0, f_rgba[:, 3] > 0)
    if not spectrum:
        assert not np.array_equal(d_rgb, f_rgb)
    s.close()


def test_double_sums_slabs():
    """Slabs put together equal the whole image with double sums too."""
    from math_b200 import tiles

    desc = scenes.cornell_3d(size=(20, 17), subdivisions=2)
    s = P.Scene(desc, "float", False)
    whole = s.painter(16, 5, seed=2)
    whole.run(2)
    ref, _ = whole.images()
    parts = []
    for rank in range(3):
        p = s.painter(16, 5, seed=2, slab=tiles.slab_rows(17, rank, 3))
        p.run(2)
        parts.append(p.images()[0])
        p.close()
    assert np.array_equal(tiles.assemble(parts), ref)
    whole.close()
    with pytest.raises(P.PainterError):
        s.painter(16, 5, pixel_sums="half")
    s.close()
