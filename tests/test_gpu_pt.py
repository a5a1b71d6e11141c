"""Parity of the GPU path tracer (integrator "pt") with the reference's PT
integrator (src/painter/integrators/pt/pt.cpp, direct_lighting.cpp,
com/surface_sample.cpp).

Double precision is compared bit for bit against the committed fixtures
(tests/golden/pt.npz, made by the compiled reference): the same sample
points and per-path random streams as the BPT painter, next-event
estimation with the power heuristic for every light, Russian roulette on
the luminance of all colour channels.  The image estimator is the one the
BPT tests pin, so its bar is theirs.
"""

import numpy as np
import pytest

from math_b200 import scenes

pytestmark = pytest.mark.gpu

SMALL = {
    "cornell3d": (lambda: scenes.cornell_3d(size=(16, 16), subdivisions=3), False, 16),
    "cornell4d": (lambda: scenes.cornell_4d(size=(6, 6, 6), points=600), True, 8),
    "cornell5d": (lambda: scenes.cornell_5d(size=(4, 4, 4, 4), points=200), False, 16),
    "sphere4d": (lambda: scenes.sphere_4d(size=(8, 8, 8), points=2000, buckets=4), False, 16),
}


def mesh_data(g, prefix=""):
    return [{"vertices": g[f"{prefix}mesh_vertices"], "normals": g[f"{prefix}mesh_normals"],
             "facets": g[f"{prefix}mesh_facets"], "facet_material": g[f"{prefix}mesh_facet_material"],
             "material_params": g[f"{prefix}mesh_material_params"],
             "material_colors": g[f"{prefix}mesh_material_colors"]}]


def scene_of(painter, golden, name, precision="double"):
    make, spectrum, spp = SMALL[name]
    if name == "sphere4d":
        data = mesh_data(golden("pt"), "sphere4d_")
    else:
        data = mesh_data(golden(name))
    return painter.Scene(make(), precision, spectrum, mesh_data=data), spp


def rel_rmse(x, ref):
    return float(np.sqrt(((x - ref) ** 2).sum() / (ref ** 2).sum()))


@pytest.mark.parametrize("name", list(SMALL))
def test_pt_samples_bit_exact(painter, golden, name):
    """Every per-path colour of a seeded pass equals the reference's pt()
    output for the same stream, bit for bit: parallelotope lights (3-, 4-
    and 5-space, RGB and 64-bin spectrum) and a ball light (4-space)."""
    g = golden("pt")
    s, spp = scene_of(painter, golden, name)
    p = s.painter(spp, 0, seed=1, integrator="pt")
    p.run(1)
    _, colors, valid = p.samples()
    assert np.array_equal(valid, g[f"{name}_valid"])
    assert np.array_equal(colors, g[f"{name}_colors"])
    stats = p.statistics()
    assert stats["ray_count"] > stats["sample_count"]
    assert stats["kernel_launches"] == 3  # sample points, paths, pixel accumulation


@pytest.mark.parametrize("name", ["cornell3d", "sphere4d"])
def test_pt_image_matches_reference_estimator(painter, golden, name):
    g = golden("pt")
    s, spp = scene_of(painter, golden, name)
    p = s.painter(spp, 0, seed=1, integrator="pt")
    p.run(1)
    rgb, rgba = p.images()
    ref = g[f"{name}_rgb"]
    assert rel_rmse(rgb, ref) < 1e-6
    assert np.isclose(rgb, ref, rtol=1e-5, atol=1e-9).all()
    assert (rgb == ref).all(axis=1).mean() >= 0.95
    assert np.isclose(rgba, g[f"{name}_rgba"], rtol=1e-5, atol=1e-9).all()


def test_pt_float_against_double_reference(painter, oracle_lib):
    """Single precision PT against the double-precision reference PT image
    of the same scene and seed: relative RMSE within 2%."""
    desc = scenes.cornell_3d(size=(32, 32), subdivisions=3)
    o = oracle_lib.Scene(desc, "double", False)
    o.set_integrator("pt")
    ref, _ = o.render_image(64, 5, seed=7, passes=4)
    s = painter.Scene(desc, "float", False)
    p = s.painter(64, 5, seed=7, integrator="pt")
    p.run(4)
    rgb, _ = p.images()
    assert rel_rmse(rgb, ref) < 0.02


def test_pt_errors(painter):
    desc = scenes.cornell_3d(size=(4, 4), subdivisions=1)
    s = painter.Scene(desc, "double", False)
    with pytest.raises(painter.PainterError, match="Unknown integrator"):
        s.painter(4, 5, integrator="mlt")
    L = painter.lib()
    assert not L.nbpt_painter_create_integrator(s.h, 7, 4, 5, 1)
    assert "Unknown integrator" in L.nbpt_last_error().decode()
    # PT ignores the BPT depth bound
    p = s.painter(4, 0, integrator="pt")
    p.run(1)
    assert p.statistics()["pass_number"] == 1
