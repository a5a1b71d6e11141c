"""Parity at the benchmark configurations' own sizes.

1. Closest hits in FP64 on the full meshes (the 4-space Cornell box's hull of
   20,000 points on S^3, about 135k facets, and the 4-space hull of 150,000
   noisy points, 321,175 facets), against the reference's scene and mesh
   queries (the oracle) on a seeded ray set: camera rays of the projector and
   rays from random points of the scene's box in random directions, as in
   src/painter/shapes/test/spherical_mesh.h:192-240.  Bit-exact.
2. The FP32 closest-hit mismatch rate on the same rays against FP64.
3. FP32 against FP64 on the same random streams at each configuration's
   full screen: relative RMSE of the images (sqrt(sum (x - r)^2 / sum r^2)
   over pixels and channels), at most 1 %.  With the same streams a path
   differs only where float rounding turns a decision, so the RMSE measures
   what FP32 changes in the image, noise of those paths included.
"""

from __future__ import annotations

import numpy as np
import pytest

from math_b200 import painter as P
from math_b200 import scenes

pytestmark = pytest.mark.gpu


def rel_rmse(x, ref) -> float:
    x = x.astype(np.float64)
    ref = ref.astype(np.float64)
    return float(np.sqrt(((x - ref) ** 2).sum() / (ref ** 2).sum()))


def seeded_rays(desc: dict, count: int, seed: int) -> np.ndarray:
    """Half camera rays through random screen points, half rays from random
    points of [-1.2, 1.2]^n in random directions."""
    n = desc["n"]
    rng = np.random.default_rng(seed)
    m = count // 2
    p = desc["projector"]
    org = np.array(p["org"], np.float64)
    axes = np.array(p["axes"], np.float64)
    size = np.array(p["size"], np.float64)
    fwd = np.array(p["dir"], np.float64)
    u = rng.uniform(-0.5, 0.5, (m, n - 1))
    if p["type"] == "perspective":
        half = np.tan(np.radians(p["fov"]) / 2)
        d = fwd + (u * (size / size.max()) * 2 * half) @ axes
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        cam = np.concatenate([np.repeat(org[None], m, 0), d], axis=1)
    else:
        o = org + (u * size * p["units_per_pixel"]) @ axes
        cam = np.concatenate([o, np.repeat(fwd[None], m, 0)], axis=1)
    o = rng.uniform(-1.2, 1.2, (count - m, n))
    d = rng.normal(size=(count - m, n))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([cam, np.concatenate([o, d], axis=1)], axis=0)


FULL_MESHES = {
    "4-space Cornell box, hull of 20000 points": lambda: scenes.cornell_4d(size=(8, 8, 8), points=20000),
    "4-space hull of 150000 noisy points": lambda: scenes.sphere_4d(size=(8, 8, 8), points=150000),
}


@pytest.fixture(scope="module", params=list(FULL_MESHES))
def full_mesh(request):
    return request.param, FULL_MESHES[request.param]()


def test_fp64_closest_hits_bit_exact_on_full_meshes(painter, oracle_lib, full_mesh):
    name, desc = full_mesh
    o = oracle_lib.Scene(desc, "double", False)
    s = painter.Scene(desc, "double", False)
    rays = seeded_rays(desc, 1 << 16, 21)
    hit, t_ref, p_ref, _ = o.scene_trace(rays)
    kind, index, t, point = s.trace(rays)
    assert np.array_equal(kind > 0, hit)
    assert np.array_equal(t[hit], t_ref[hit])
    assert np.array_equal(point[hit], p_ref[hit])
    facet = kind == 3
    assert facet.sum() > 100
    # one mesh shape: a facet hit through the scene is the mesh's own closest facet
    assert len(o.mesh_shapes) == 1
    facet_ref, _ = o.mesh_trace(rays)
    assert np.array_equal(index[facet], facet_ref[facet])
    s.close()


def test_fp32_closest_hit_mismatch_rate(painter, full_mesh):
    """FP32 traversal and intersection against FP64 on the same rays: the
    share of rays whose hit (none, shape or facet) differs.  Stated, and
    bounded at 0.1 %."""
    name, desc = full_mesh
    d64 = painter.Scene(desc, "double", False)
    d32 = painter.Scene(desc, "float", False)
    rays = seeded_rays(desc, 1 << 18, 22)
    k64, i64, t64, _ = d64.trace(rays)
    k32, i32, t32, _ = d32.trace(rays)
    differ = (k64 != k32) | ((k64 > 0) & (i64 != i32))
    rate = float(differ.mean())
    hit = (k64 > 0) & (k32 > 0) & ~differ
    dt = np.abs(t32[hit] - t64[hit]) / np.maximum(t64[hit], 1e-12)
    print(f"\n{name}: FP32 closest-hit mismatch rate {rate:.2e} over {len(rays)} rays; "
          f"median relative distance error of the matching hits {np.median(dt):.1e}")
    assert rate <= 1e-3
    assert np.median(dt) < 1e-5
    d64.close()
    d32.close()


CONFIGS = {
    # name: (scene, spectrum, samples per pixel, depth, passes at the first
    # and at the second measurement)
    "C1 3-space Cornell, 256^2, 16 spp, depth 5, RGB": (lambda: scenes.cornell_3d(), False, 16, 5, (2, 8)),
    "C2 4-space Cornell, 64^3, 16 (27) spp, depth 6, spectrum": (lambda: scenes.cornell_4d(), True, 16, 6, (2, 16)),
    "C3 4-space 321k-facet hull, 96^3, 8 spp, depth 8, RGB": (lambda: scenes.sphere_4d(), False, 8, 8, (2, 40)),
}


def same_stream_rmse(painter, jobs, passes):
    """FP32 against FP64 images of the same jobs on the same random streams,
    after each count of passes in `passes`: the relative RMSE over all the
    jobs' pixels.  A path differs between the two only where float rounding
    turns one of its decisions, so the difference is the noise of those
    paths (it falls as 1/sqrt(passes)) plus any bias of FP32 (it would not)."""
    pairs = []
    for desc, spectrum, spp, depth in jobs:
        pair = []
        for precision in ("double", "float"):
            s = painter.Scene(desc, precision, spectrum)
            pair.append((s, s.painter(spp, depth, seed=3)))
        pairs.append(pair)
    out = []
    done = 0
    for p in passes:
        num = den = 0.0
        for pair in pairs:
            images = []
            for _, painter_ in pair:
                painter_.run(p - done)
                images.append(painter_.images()[0].astype(np.float64))
            num += float(((images[1] - images[0]) ** 2).sum())
            den += float((images[0] ** 2).sum())
        done = p
        out.append(float(np.sqrt(num / den)))
    for pair in pairs:
        for s, painter_ in pair:
            painter_.close()
            s.close()
    return out


@pytest.mark.parametrize("name", list(CONFIGS))
def test_fp32_image_rmse_per_config(painter, name):
    make, spectrum, spp, depth, passes = CONFIGS[name]
    err = same_stream_rmse(painter, [(make(), spectrum, spp, depth)], passes)
    print(f"\n{name}: FP32 vs FP64, same streams: relative RMSE "
          + ", ".join(f"{e:.4f} after {p} passes" for e, p in zip(err, passes)))
    # noise, not bias: more passes shrink it
    assert err[1] < err[0]
    assert err[1] <= 0.01


def test_fp32_image_rmse_mixed_batch_subset(painter):
    """Eight jobs of the mixed-scene batch (seed 4) at full size, FP32 against
    FP64 on the same streams, the relative RMSE over all their pixels."""
    jobs = scenes.mixed_batch(64, seed=4, select=[1, 5, 9, 12, 22, 27, 41, 60])
    passes = (2, 32)
    err = same_stream_rmse(painter, [(j["desc"], False, j["spp"], j["max_depth"]) for j in jobs], passes)
    print("\nmixed batch, 8 jobs: FP32 vs FP64, same streams: relative RMSE "
          + ", ".join(f"{e:.4f} after {p} passes" for e, p in zip(err, passes)))
    assert err[1] < err[0]
    assert err[1] <= 0.01
