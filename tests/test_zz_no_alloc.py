"""nbpt_scene_trace_noalloc: ray queries through the fixed device scratch
array, called through the C ABI and compared with nbpt_scene_trace (which
allocates per call) on the same rays, twice in a row.  The two run the same
query kernel on the same inputs, so the tolerance is exact equality."""

from __future__ import annotations

import numpy as np
import pytest

from math_b200 import painter as P
from math_b200 import scenes

MAX_RAYS = 16384


def call_noalloc(scene, rays: np.ndarray, any_hit: bool):
    rays = np.ascontiguousarray(rays, dtype=np.float64).reshape(-1, 2 * scene.n)
    m = len(rays)
    kind = np.full(m, -7, np.int32)
    index = np.full(m, -7, np.int32)
    t = np.full(m, np.nan)
    point = np.full((m, scene.n), np.nan)
    r = P.lib().nbpt_scene_trace_noalloc(
        scene.h, P._p(rays, P._D), m, 1 if any_hit else 0, P._p(kind, P._I), P._p(index, P._I),
        P._p(t, P._D), P._p(point, P._D))
    return r, kind, index, t, point


def seeded_rays(n: int, count: int, seed: int) -> np.ndarray:
    """Rays from points inside the box [-1, 1]^n in uniformly random directions."""
    rng = np.random.default_rng(seed)
    org = rng.uniform(-0.9, 0.9, (count, n))
    d = rng.normal(size=(count, n))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([org, d], axis=1)


CASES = {
    "cornell3d": (lambda: scenes.cornell_3d(size=(16, 16), subdivisions=3), False, 3),
    "cornell4d": (lambda: scenes.cornell_4d(size=(6, 6, 6), points=600), True, 4),
    "cornell5d": (lambda: scenes.cornell_5d(size=(4, 4, 4, 4), points=200), False, 5),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("count", [1, 4096, MAX_RAYS])
def test_noalloc_trace_matches_allocating_trace(name, count):
    if P.device_count() < 1:
        pytest.fail("no CUDA device visible to the painter library")
    make, spectrum, n = CASES[name]
    scene = P.Scene(make(), "float", spectrum)
    rays = seeded_rays(n, count, seed=11 + count)
    kind, index, t, point = scene.trace(rays)
    any_ref = scene.trace(rays, any_hit=True)
    assert count == 1 or (kind > 0).any()  # the box has an open side: one ray may escape
    for _ in range(2):  # two calls in a row through the same scratch
        r, k2, i2, t2, p2 = call_noalloc(scene, rays, any_hit=False)
        assert r == 0, P.lib().nbpt_last_error()
        assert np.array_equal(k2, kind)
        assert np.array_equal(i2, index)
        assert np.array_equal(t2, t)
        assert np.array_equal(p2, point)
        r, ka, _, _, _ = call_noalloc(scene, rays, any_hit=True)
        assert r == 0, P.lib().nbpt_last_error()
        assert np.array_equal(ka.astype(bool), any_ref)
    scene.close()


@pytest.mark.gpu
def test_noalloc_trace_rejects_more_rays_than_its_scratch():
    if P.device_count() < 1:
        pytest.fail("no CUDA device visible to the painter library")
    make, spectrum, n = CASES["cornell3d"]
    scene = P.Scene(make(), "float", spectrum)
    rays = seeded_rays(n, MAX_RAYS + 1, seed=5)
    r, kind, _, _, _ = call_noalloc(scene, rays, any_hit=False)
    assert r == -1  # NBPT_ERROR
    assert b"16384" in P.lib().nbpt_last_error()
    assert (kind == -7).all()  # nothing written
    # zero rays: nothing to do
    r, _, _, _, _ = call_noalloc(scene, rays[:0], any_hit=False)
    assert r == 0
    # the scratch still serves a full call afterwards
    r, k2, _, _, _ = call_noalloc(scene, rays[:MAX_RAYS], any_hit=False)
    assert r == 0
    assert np.array_equal(k2, scene.trace(rays[:MAX_RAYS])[0])
    scene.close()
