"""The CPU restatement (oracle/port.py) against the known-answer vectors of
the reference's own tests and against the compiled reference."""

import json

import numpy as np
import pytest

from oracle import port

from conftest import GOLDEN


@pytest.fixture(scope="module")
def kat():
    return json.loads((GOLDEN / "reference_kat.json").read_text())


def test_paintbrush_order(kat):
    for case in kat["paintbrush"]:
        got = port.paintbrush_pixels(case["size"], case["paint_height"])
        assert [list(p) for p in got] == case["pixels"], case["source"]


def test_paintbrush_covers_screen():
    for size in ([5, 7], [3, 4, 2], [20, 1, 3]):
        got = port.paintbrush_pixels(size, 3)
        assert len(got) == int(np.prod(size))
        assert len(set(got)) == len(got)


def test_background_sample_creation(kat):
    for case in kat["background_samples"]:
        weights = [w for w, v in zip(case["weights"], case["valid"]) if not v and w > 0]
        kept, summed, full = port.create_samples(weights, case["count"])
        assert full == case["full"], case["source"]
        assert [weights[i] for i in kept] == case["kept_weights"], case["source"]
        if full:
            assert sum(weights[i] for i in summed) == pytest.approx(case["weight_sum"]), case["source"]


def test_color_sample_creation(kat):
    for case in kat["color_samples"]:
        items = [(w, c) for w, c in zip(case["weights"], case["colors"]) if c is not None and w > 0]
        keys = [np.float32(w) * np.float32(port.luminance_rgb([c, c, c])) for w, c in items]
        kept, summed, full = port.create_samples(keys, case["count"])
        assert full == case["full"], case["source"]
        assert [list(items[i]) for i in kept] == [list(x) for x in case["kept"]], case["source"]
        if full:
            assert sorted(list(items[i]) for i in summed) == sorted(list(x) for x in case["summed"]), case["source"]


def test_rng_restatement_matches_golden(golden):
    g = golden("rng")
    for i in range(4):
        words = [int(x) for x in g[f"seed_{i}"]]
        pcg = port.Pcg(words)
        assert np.array_equal([pcg() for _ in range(64)], g[f"pcg_{i}"])
        pcg = port.Pcg(words)
        assert np.array_equal([pcg.canonical(True) for _ in range(64)], g[f"canonical_double_{i}"])
        pcg = port.Pcg(words)
        assert np.array_equal([pcg.canonical(False) for _ in range(64)], g[f"canonical_float_{i}"])
        for dim in (2, 3):
            for dbl in (True, False):
                got = port.sj_points(dim, 16, words, dbl)
                assert np.array_equal(got, g[f"sj_{dim}_{int(dbl)}_{i}"])


def test_simplex_restatement_matches_golden(golden):
    g = golden("cornell3d")
    v = g["mesh_vertices"][g["mesh_facets"]]
    planes = port.simplex_planes(v)
    ref = g["mesh_planes"]
    # the facet plane may be reversed to follow the vertex normals
    # (src/painter/shapes/mesh/facet.cpp:113-118)
    sign = np.sign(np.einsum("fi,fi->f", planes[:, 0, :3], ref[:, 0, :3]))[:, None]
    assert np.allclose(planes[:, 0] * sign, ref[:, 0], rtol=1e-9, atol=1e-12)
    assert np.allclose(planes[:, 1:], ref[:, 1:], rtol=1e-9, atol=1e-12)


def test_simplex_intersection_restatement(golden):
    g = golden("cornell3d")
    rays = g["rays"][:512]
    # the reference's Ray normalises its direction (src/numerical/ray.h)
    d = rays[:, 3:] / np.linalg.norm(rays[:, 3:], axis=1, keepdims=True)
    t = port.simplex_intersect(g["mesh_planes"], rays[:, :3], d)
    t_masked = np.where(t > 0, t, np.inf)
    facet = np.where(np.isfinite(t_masked.min(axis=1)), t_masked.argmin(axis=1), -1)
    assert np.array_equal(facet, g["ray_facet"][:512])
    hit = facet >= 0
    assert np.allclose(t_masked.min(axis=1)[hit], g["ray_t"][:512][hit], rtol=1e-12)
