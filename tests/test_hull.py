"""The scene generators' convex hulls (math_b200.scenes.convex_hull_mesh)
against the reference's own compute_convex_hull (src/geometry/core/
convex_hull.h:95-98), compiled from its sources into the oracle
(oracle/_ref/libnbpt_hull.so; 5-space computes with GMP integers through
the system's libgmp).

The facet sets are equal, as sets of vertex-index sets, for the benchmark
hulls: the 4-space Cornell sphere (20,000 points), the C3 4-space sphere
(150,000 noisy points, 321k facets), every 3- and 4-space hull of the mixed
batch up to 25,000 points and its 5-space hulls up to 3,500 points (the
reference's 5-space hull takes about 2 s per 1,000 points here)."""

from __future__ import annotations

import numpy as np
import pytest

from math_b200 import scenes


@pytest.fixture(scope="module")
def hull_lib():
    from oracle import oracle

    if not oracle.hull_available():
        pytest.skip("hull library not built (make -C oracle hull)")
    return oracle


def facet_set(facets: np.ndarray) -> set:
    return set(map(tuple, np.sort(np.asarray(facets), axis=1).tolist()))


def check(hull_lib, points):
    _, f = scenes.convex_hull_mesh(points)
    ref = hull_lib.convex_hull(points)
    assert len(f) == len(ref)
    assert facet_set(f) == facet_set(ref)
    return len(f)


def test_integer_grid_matches_the_reference_rounding():
    p = np.array([[0.0, 0.0, 0.0], [1.0, 0.5, 0.25], [0.5, 2.0, 1.0]], np.float32)
    q = scenes.hull_integer_points(p)
    m = (1 << 30) - 1
    assert q.max() == m and q.min() == 0
    # extent 2 on the second axis: 1.0 -> (2^30 - 1) / 2 rounded half away from zero
    assert q[1, 0] == np.floor(m / 2 + 0.5)
    assert (q == np.floor(q)).all()


@pytest.mark.parametrize("n, count, seed", [(3, 3000, 1), (4, 3000, 1), (5, 2000, 1)])
def test_small_hulls(hull_lib, n, count, seed):
    check(hull_lib, scenes.sphere_points(n, count, seed))


def test_duplicate_points_keep_the_first(hull_lib):
    p = scenes.sphere_points(3, 500, 4)
    p = np.concatenate([p, p[:50]])
    _, f = scenes.convex_hull_mesh(p)
    assert f.max() < 500
    check(hull_lib, p)


def test_cornell_4d_sphere(hull_lib):
    assert check(hull_lib, scenes.sphere_points(4, 20000, 2)) > 130000


def test_sphere_4d_noisy(hull_lib):
    assert check(hull_lib, scenes.sphere_points(4, 150000, 3, noise=0.002)) > 300000


def test_mixed_batch_hulls(hull_lib):
    checked = 0
    for _, n, points, seed in scenes.mixed_batch_hulls():
        if (n in (3, 4) and points <= 25000) or (n == 5 and points <= 3500):
            check(hull_lib, scenes.sphere_points(n, points, seed))
            checked += 1
    assert checked >= 18
