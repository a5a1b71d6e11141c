"""Parity of the CUDA path with the reference painter.

Double precision is compared bit for bit: the GPU kernels follow the
reference's operation order with no multiply-add contraction, consume each
path's random stream in the reference's order, and so reproduce the
reference's per-sample colours exactly.  Single precision is compared with
the double-precision reference image through relative RMSE.

The reference is the committed golden fixtures (made by the CPU oracle,
tests/golden/make_golden.py) and, where it is built, the live oracle.
"""

import numpy as np
import pytest

from math_b200 import scenes

pytestmark = pytest.mark.gpu

SMALL = {
    "cornell3d": (lambda: scenes.cornell_3d(size=(16, 16), subdivisions=3), False),
    "cornell4d": (lambda: scenes.cornell_4d(size=(6, 6, 6), points=600), True),
    "cornell5d": (lambda: scenes.cornell_5d(size=(4, 4, 4, 4), points=200), False),
}


def mesh_data(g):
    return [{"vertices": g["mesh_vertices"], "normals": g["mesh_normals"], "facets": g["mesh_facets"],
             "facet_material": g["mesh_facet_material"], "material_params": g["mesh_material_params"],
             "material_colors": g["mesh_material_colors"]}]


def rel_rmse(x, ref):
    return float(np.sqrt(((x - ref) ** 2).sum() / (ref ** 2).sum()))


# --------------------------------------------------------------------------
# random streams


def test_rng_streams_bit_exact(painter, golden):
    g = golden("rng")
    for i in range(4):
        words = [int(x) for x in g[f"seed_{i}"]]
        assert np.array_equal(painter.test_pcg(words, 64), g[f"pcg_{i}"])
        assert np.array_equal(painter.test_canonical(words, 64, True), g[f"canonical_double_{i}"])
        assert np.array_equal(painter.test_canonical(words, 64, False), g[f"canonical_float_{i}"])
        for dim, spp in ((2, 16), (3, 16), (4, 81)):
            for dbl in (True, False):
                assert np.array_equal(painter.test_sj_points(dim, spp, words, dbl), g[f"sj_{dim}_{int(dbl)}_{i}"])


# --------------------------------------------------------------------------
# geometry


@pytest.mark.parametrize("name", ["cornell3d", "cornell4d"])
def test_facet_records_and_bvh_bit_exact(painter, golden, name):
    """Facet hyperplanes (set up in double on the GPU) and the BVH (built on
    the host) equal the reference's own, record for record."""
    g = golden(name)
    make, spectrum = SMALL[name]
    s = painter.Scene(make(), "double", spectrum, mesh_data=mesh_data(g))
    e = s.mesh_export(0)
    assert np.array_equal(e["planes"], g["mesh_planes"])
    assert np.array_equal(e["node_lo"], g["mesh_node_bounds"][:, 0])
    assert np.array_equal(e["node_hi"], g["mesh_node_bounds"][:, 1])
    assert np.array_equal(e["node_info"], g["mesh_node_info"])
    assert np.array_equal(e["indices"], g["mesh_indices"])


@pytest.mark.parametrize("name", ["cornell3d", "cornell4d", "cornell5d"])
def test_closest_hit_bit_exact(painter, golden, name):
    """Closest hits of a seeded ray set through the whole scene: hit flag,
    distance and point equal the reference's; facet hits name the same facet."""
    g = golden(name)
    make, spectrum = SMALL[name]
    s = painter.Scene(make(), "double", spectrum, mesh_data=mesh_data(g))
    kind, index, t, point = s.trace(g["rays"])
    hit = kind > 0
    assert np.array_equal(hit, g["scene_hit"])
    assert np.array_equal(t[hit], g["scene_t"][hit])
    assert np.array_equal(point[hit], g["scene_point"][hit])
    facet = kind == 3
    mesh_hit = g["ray_facet"] >= 0
    # a facet hit through the scene is the mesh's own closest facet
    assert np.array_equal(index[facet], g["ray_facet"][facet])
    assert facet.sum() > 0 and mesh_hit.sum() >= facet.sum()


def test_own_ingestion_closest_hit(painter, oracle_lib):
    """The library's own mesh ingestion (vertex transform, its BVH build)
    gives the reference's closest hits on the 20,480-triangle icosphere."""
    desc = scenes.cornell_3d(size=(8, 8), subdivisions=5)
    o = oracle_lib.Scene(desc, "double", False)
    s = painter.Scene(desc, "double", False)
    rng = np.random.default_rng(3)
    rays = np.concatenate([rng.uniform(-1, 1, (20000, 3)), rng.normal(size=(20000, 3))], axis=1)
    hit, t_ref, p_ref, _ = o.scene_trace(rays)
    kind, index, t, point = s.trace(rays)
    assert np.array_equal(kind > 0, hit)
    assert np.array_equal(t[hit], t_ref[hit])
    facet_ref, _ = o.mesh_trace(rays)
    facet = kind == 3
    assert np.array_equal(index[facet], facet_ref[facet])
    e = s.mesh_export(0)
    m = o.mesh_dump()
    assert np.array_equal(e["node_info"], m["node_info"])
    assert np.array_equal(e["indices"], m["indices"])


# --------------------------------------------------------------------------
# BRDF and lights


def test_brdf_and_sampling_bit_exact(painter, oracle_lib):
    desc = scenes.cornell_4d(size=(4, 4, 4), points=200)
    o = oracle_lib.Scene(desc, "double", True)
    s = painter.Scene(desc, "double", True)
    rng = np.random.default_rng(11)
    # material of shape 0 (the first wall) and of the rotated parallelotope
    for material, shape in ((0, desc["shapes"][0]), (8, desc["shapes"][8])):
        for k in range(16):
            n = rng.normal(size=4)
            n /= np.linalg.norm(n)
            v = rng.normal(size=4)
            v /= np.linalg.norm(v)
            v = v if v @ n > 0 else -v
            l = rng.normal(size=4)
            l /= np.linalg.norm(l)
            f, pdf = s.brdf(material, n, v, l)
            fo, pdfo = o.brdf(shape["metalness"], shape["roughness"], shape["color"], n, v, l)
            assert np.array_equal(f, fo) and pdf == pdfo
            ls, pdfs, fs = s.brdf_sample(material, n, v, [k, 5])
            lo, pdfo2, fo2 = o.brdf_sample(shape["metalness"], shape["roughness"], shape["color"], n, v, [k, 5])
            assert pdfs == pdfo2
            if pdfs > 0:
                assert np.array_equal(ls, lo) and np.array_equal(fs, fo2)


def test_light_samples_bit_exact(painter, oracle_lib):
    for desc, spectrum in ((scenes.cornell_3d(size=(4, 4), subdivisions=1), False),
                           (scenes.sphere_4d(size=(4, 4, 4), points=500, buckets=2), False)):
        o = oracle_lib.Scene(desc, "double", spectrum)
        s = painter.Scene(desc, "double", spectrum)
        n = desc["n"]
        for k in range(8):
            a, ra = s.light_sample(0, "leave", [3, k])
            b, rb = o.light_sample(0, "leave", [3, k])
            assert np.array_equal(a, b) and np.array_equal(ra, rb)
            p = np.full(n, -0.2)
            a, ra = s.light_sample(0, "arrive", [4, k], point=p)
            b, rb = o.light_sample(0, "arrive", [4, k], point=p)
            assert np.array_equal(a[: n + 2], b[: n + 2]) and np.array_equal(ra, rb)


# --------------------------------------------------------------------------
# paths


@pytest.mark.parametrize("name", ["cornell3d", "cornell4d", "cornell5d"])
def test_path_samples_bit_exact(painter, golden, name):
    """Every per-path colour of a seeded pass equals the reference's bpt()
    output for the same stream, bit for bit, in 3-, 4- (64-bin spectrum) and
    5-space."""
    g = golden(name)
    make, spectrum = SMALL[name]
    s = painter.Scene(make(), "double", spectrum, mesh_data=mesh_data(g))
    p = s.painter(int(g["spp"]), int(g["depth"]), seed=1)
    p.run(1)
    points, colors, valid = p.samples()
    assert np.array_equal(points, g["points"])
    assert np.array_equal(valid, g["valid"])
    assert np.array_equal(colors, g["colors"])
    stats = p.statistics()
    assert stats["sample_count"] == g["colors"].shape[0] * g["colors"].shape[1]
    assert stats["ray_count"] > stats["sample_count"]


@pytest.mark.parametrize("name", ["cornell3d", "cornell4d", "cornell5d"])
def test_image_matches_reference_estimator(painter, golden, name):
    """The filtered, trimmed pixel estimator: from identical samples, the
    image equals the reference's Pixels::images (sources merged into each
    pixel in increasing pixel index).  Held-out selection, merge order and
    float sums follow the reference step for step; the filter weights use
    the device's exp, which may differ from the host's in the last bit, so
    the bar is: nearly every pixel bit-identical, the rest within 1e-5."""
    g = golden(name)
    make, spectrum = SMALL[name]
    s = painter.Scene(make(), "double", spectrum, mesh_data=mesh_data(g))
    p = s.painter(int(g["spp"]), int(g["depth"]), seed=1)
    p.run(1)
    rgb, rgba = p.images()
    ref = g["rgb"]
    assert rel_rmse(rgb, ref) < 1e-6
    assert np.isclose(rgb, ref, rtol=1e-5, atol=1e-9).all()
    assert (rgb == ref).all(axis=1).mean() >= 0.95
    assert np.isclose(rgba, g["rgba"], rtol=1e-5, atol=1e-9).all()


@pytest.mark.parametrize("name", list(SMALL))
def test_own_ingestion_paths(painter, oracle_lib, name):
    """The full drop-in path, with nothing injected: mesh objects ingested by
    the library (used points, vertex normals with the reference's signs,
    transforms), its own BVH and FP64 facet set-up, against the reference
    painter on the same scene description.  Every sample is bit-identical;
    the image as in test_image_matches_reference_estimator."""
    make, spectrum = SMALL[name]
    desc = make()
    o = oracle_lib.Scene(desc, "double", spectrum)
    s = painter.Scene(desc, "double", spectrum)
    p = s.painter(16, 5, seed=1)
    p.run(1)
    _, colors, valid = p.samples()
    _, ref, ref_valid = o.render_samples(16, 5, seed=1)
    assert np.array_equal(valid, ref_valid)
    assert np.array_equal(colors, ref)
    rgb, _ = p.images()
    ref_rgb, _ = o.render_image(16, 5, seed=1)
    assert rel_rmse(rgb, ref_rgb) < 1e-6
    assert np.isclose(rgb, ref_rgb, rtol=1e-5, atol=1e-9).all()
    assert (rgb == ref_rgb).all(axis=1).mean() >= 0.95


def test_float_path_rmse_against_double_reference(painter, oracle_lib):
    """Single precision (traversal, intersection, BRDF and MIS in float;
    facet set-up and the per-pixel radiance sums in double) against the
    double-precision reference image of the same scene: relative RMSE
    within 1%."""
    desc = scenes.cornell_3d(size=(32, 32), subdivisions=3)
    o = oracle_lib.Scene(desc, "double", False)
    ref, _ = o.render_image(64, 5, seed=7, passes=4)
    s = painter.Scene(desc, "float", False)
    p = s.painter(64, 5, seed=7)
    p.run(4)
    rgb, _ = p.images()
    # same seed, same estimator: the difference is float rounding plus the
    # paths it re-routes; both images hold 256 samples per pixel
    assert rel_rmse(rgb, ref) < 0.01


def test_passes_accumulate(painter, golden):
    g = golden("cornell3d")
    make, spectrum = SMALL["cornell3d"]
    s = painter.Scene(make(), "double", spectrum, mesh_data=mesh_data(g))
    p = s.painter(16, 5, seed=1)
    p.run(1)
    one, _ = p.images()
    p.run(3)
    four, _ = p.images()
    assert p.statistics()["pass_number"] == 4
    assert not np.array_equal(one, four)
    assert np.isfinite(four).all()


# --------------------------------------------------------------------------
# error behaviour


def test_errors(painter):
    desc = scenes.cornell_3d(size=(4, 4), subdivisions=1)
    s = painter.Scene(desc, "double", False)
    with pytest.raises(painter.PainterError, match="samples per pixel"):
        s.painter(0, 5)
    with pytest.raises(painter.PainterError, match="maximum depth"):
        s.painter(4, 9)
    bad = dict(desc)
    bad["background"] = [0.1, 0.1, 0.1]
    with pytest.raises(painter.PainterError, match="background"):
        painter.Scene(bad, "double", False)
    bad = dict(desc)
    bad["lights"] = []
    with pytest.raises(painter.PainterError, match="No light sources"):
        painter.Scene(bad, "double", False)


def test_build_seconds(painter):
    """The scene reports where its build time went (mesh ingestion, BVH,
    the rest of finalize); the parts add up to the total."""
    desc = scenes.cornell_3d(size=(8, 8), subdivisions=2)
    s = painter.Scene(desc, "float", False)
    b = s.build_seconds()
    assert set(b) == {"ingest", "bvh", "upload", "total"}
    assert all(v >= 0 for v in b.values())
    assert b["bvh"] > 0 and b["total"] > 0
    assert abs(b["ingest"] + b["bvh"] + b["upload"] - b["total"]) < 1e-9


@pytest.mark.parametrize("name", list(SMALL))
@pytest.mark.parametrize("integrator", ["bpt", "pt"])
def test_flat_shading_paths_bit_exact(painter, oracle_lib, name, integrator):
    """create_painter's flat_shading (bpt<true> / pt<true>: the geometric
    normal shades, src/painter/integrators/com/normals.h:45-64): every sample
    equals the reference's, and differs from smooth shading where the
    sphere's interpolated normals were used."""
    make, spectrum = SMALL[name]
    desc = make()
    o = oracle_lib.Scene(desc, "double", spectrum)
    o.set_integrator(integrator)
    o.set_flat_shading(True)
    s = painter.Scene(desc, "double", spectrum)
    p = s.painter(16, 5, seed=1, integrator=integrator, flat_shading=True)
    p.run(1)
    _, colors, valid = p.samples()
    _, ref, ref_valid = o.render_samples(16, 5, seed=1)
    assert np.array_equal(valid, ref_valid)
    assert np.array_equal(colors, ref)
    smooth = s.painter(16, 5, seed=1, integrator=integrator)
    smooth.run(1)
    assert not np.array_equal(smooth.samples()[1], colors)
