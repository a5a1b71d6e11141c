"""Synthetic scene descriptions for the n-dimensional bidirectional path tracer.

A scene description is a plain dict that both the accelerated library
(`math_b200.painter`) and the CPU oracle (`oracle/oracle.py`) turn into a scene
through their own constructors, so that both render exactly the same geometry:

    {
      "n": 3 | 4 | 5,                      space dimension
      "shapes": [                          in creation order
        {"type": "hyperplane_parallelotope", "metalness", "roughness",
         "color": [r, g, b], "alpha", "org": [n], "vectors": [n-1][n]},
        {"type": "parallelotope", ... "vectors": [n][n]},
        {"type": "mesh", "objects": [
            {"points": float32 [V, n], "facets": int32 [F, n],
             "matrix": [(n+1)][(n+1)], "metalness", "roughness",
             "color": [r, g, b], "alpha"}, ...]},
            (or {"file": an OBJ / STL path, "matrix", "metalness", ...} in
             place of "points" and "facets")
      ],
      "lights": [                          in creation order
        {"type": "parallelotope", "shape": index of a hyperplane_parallelotope,
         "direction": [n], "radiance": [r, g, b]},
        {"type": "ball", "center": [n], "direction": [n], "radius",
         "radiance": [r, g, b]},
      ],
      "projector": {"type": "perspective", "org", "dir", "axes": [n-1][n],
                    "fov": degrees, "size": [n-1]}
                 | {"type": "parallel", "org", "dir", "axes",
                    "units_per_pixel", "size"},
      "background": [0, 0, 0],
    }

The constructors mirror the reference's scene API
(src/painter/shapes/hyperplane_parallelotope.h:66-77,
src/painter/shapes/parallelotope.h:65-71, src/painter/shapes/mesh.h:32-37,
src/painter/lights/parallelotope_light.h:73-83, src/painter/lights/ball_light.h:76-90,
src/painter/projectors/perspective_projector.h, parallel_projector.h,
src/painter/scenes/storage.h:40-47).  Surface colours are reflectances
(Color(r, g, b)); light colours are illuminants (Color::illuminant(r, g, b)),
as the reference's GUI creates them (src/process/painting.cpp:301).

The generators below build the benchmark workloads from fixed seeds: there is
no external dataset, every input is synthetic.
"""

from __future__ import annotations

import math

import numpy as np

# --------------------------------------------------------------------------
# meshes


def icosphere(subdivisions: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere: 20 * 4**subdivisions triangles (5 -> 20,480)."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = [
        (-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0),
        (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
        (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1),
    ]
    f = [
        (0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
        (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
        (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
        (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1),
    ]
    vertices = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in v]
    faces = list(f)
    for _ in range(subdivisions):
        cache: dict[tuple[int, int], int] = {}

        def mid(a: int, b: int) -> int:
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                p = vertices[a] + vertices[b]
                vertices.append(p / np.linalg.norm(p))
                cache[key] = len(vertices) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.asarray(vertices, dtype=np.float32), np.asarray(faces, dtype=np.int32)


def sphere_points(n: int, count: int, seed: int, noise: float = 0.0) -> np.ndarray:
    """`count` points uniform on the unit (n-1)-sphere, optionally with
    Gaussian radial noise of standard deviation `noise`."""
    rng = np.random.default_rng(seed)
    p = rng.normal(size=(count, n))
    p /= np.linalg.norm(p, axis=1, keepdims=True)
    if noise > 0:
        p *= (1.0 + noise * rng.normal(size=(count, 1)))
    return p.astype(np.float32)


def hull_integer_points(points: np.ndarray) -> np.ndarray:
    """The integer points the reference's convex hull works on
    (src/geometry/core/convex_hull/source_points.h:40-100): float points
    shifted by their per-axis minimum and scaled so the largest extent is
    2^30 - 1, the product taken in double and rounded to the nearest integer
    (halves away from zero).  Returned as float64 (exact: 30 bits)."""
    p = np.asarray(points, dtype=np.float32)
    lo = p.min(axis=0)
    hi = p.max(axis=0)
    extent = float(np.max(np.abs(hi - lo)))  # float subtraction, as the reference's Vector<N, float>
    if not extent != 0:
        raise ValueError("no distinct points")
    scale = float((1 << 30) - 1) / extent
    x = (p - lo).astype(np.float64) * scale  # float difference, double product
    r = np.floor(x)
    return r + (x - r >= 0.5)


def convex_hull_mesh(points: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Boundary facets ((n-1)-simplices) of the convex hull of `points`,
    the facet set of the reference's compute_convex_hull
    (src/geometry/core/convex_hull.h:95-98).

    The reference computes the hull exactly on the points rounded to a
    30-bit integer grid (hull_integer_points), keeping the first of points
    that round to the same integer point.  Qhull on those integer points
    finds the same facets: a double-precision hull of the unrounded points
    differs from it by a few facets wherever nearly coplanar points are
    split the other way by the rounding (tests/test_hull.py checks the
    3-, 4- and 5-space benchmark hulls against the reference's own).  Facet vertices are
    indices into `points`; the vertex order inside a facet does not matter
    to the painter, which orients normals towards the ray."""
    from scipy.spatial import ConvexHull

    q = hull_integer_points(points)
    _, first = np.unique(q, axis=0, return_index=True)
    first = np.sort(first)
    hull = ConvexHull(q[first])
    return np.asarray(points, dtype=np.float32), first[hull.simplices].astype(np.int32)


def transform_matrix(n: int, scale: float, center) -> list[list[float]]:
    m = np.eye(n + 1)
    for i in range(n):
        m[i, i] = scale
        m[i, n] = center[i]
    return m.tolist()


def random_rotation(n: int, seed: int) -> np.ndarray:
    """A rotation (det +1) drawn from the Haar measure on SO(n)."""
    rng = np.random.default_rng(seed)
    q, r = np.linalg.qr(rng.normal(size=(n, n)))
    q = q * np.sign(np.diag(r))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


# --------------------------------------------------------------------------
# building blocks


def _unit(n: int, i: int, s: float = 1.0) -> list[float]:
    v = [0.0] * n
    v[i] = s
    return v


def box_walls(n: int, half: float, colors: dict, open_axis: int, open_side: int) -> list[dict]:
    """Flat (n-1)-parallelotope faces of the cube [-half, half]^n except the
    face on side `open_side` (-1 or +1) of axis `open_axis`.  Walls are
    diffuse: metalness 0, roughness 1 (the reference has no Lambertian
    material; this is how its Cornell box makes matte walls,
    src/painter/scenes/cornell_box.cpp:198-200)."""
    walls = []
    for axis in range(n):
        for side in (-1, 1):
            if axis == open_axis and side == open_side:
                continue
            org = [-half] * n
            org[axis] = side * half
            vectors = [_unit(n, k, 2 * half) for k in range(n) if k != axis]
            walls.append({
                "type": "hyperplane_parallelotope",
                "metalness": 0.0, "roughness": 1.0,
                "color": list(colors.get((axis, side), colors["default"])),
                "alpha": 1.0, "org": org, "vectors": vectors,
            })
    return walls


def ceiling_light(n: int, half: float, size: float, up_axis: int, radiance: float) -> tuple[dict, dict]:
    """An (n-1)-parallelotope area light of edge `size` just below the
    ceiling (the face +half of `up_axis`), facing down, and its carrier."""
    org = [-size / 2] * n
    org[up_axis] = half - 1e-3
    vectors = [_unit(n, k, size) for k in range(n) if k != up_axis]
    carrier = {
        "type": "hyperplane_parallelotope", "metalness": 0.0, "roughness": 1.0,
        "color": [1.0, 1.0, 1.0], "alpha": 1.0, "org": org, "vectors": vectors,
    }
    light = {"type": "parallelotope", "direction": _unit(n, up_axis, -1.0),
             "radiance": [radiance] * 3}
    return carrier, light


def camera(n: int, distance: float, size, fov: float = 60.0) -> dict:
    """Perspective camera on the -x_{n-1} side looking along +x_{n-1}; the
    screen axes are x_0 .. x_{n-2}."""
    org = [0.0] * n
    org[n - 1] = -distance
    return {"type": "perspective", "org": org, "dir": _unit(n, n - 1),
            "axes": [_unit(n, k) for k in range(n - 1)], "fov": fov,
            "size": list(size)}


# --------------------------------------------------------------------------
# benchmark configurations


def cornell_3d(size=(256, 256), subdivisions: int = 5) -> dict:
    """3-space Cornell box: five 2x2 diffuse walls of albedo 0.7 (red and
    green sides), a 0.5x0.5 ceiling light of radiance 10, and an icosphere
    (20,480 triangles at 5 subdivisions) of radius 0.4 with GGX roughness 0.3."""
    n = 3
    colors = {"default": (0.7, 0.7, 0.7), (0, -1): (0.7, 0.07, 0.07), (0, 1): (0.07, 0.7, 0.07)}
    shapes = box_walls(n, 1.0, colors, open_axis=n - 1, open_side=-1)
    carrier, light = ceiling_light(n, 1.0, 0.5, up_axis=1, radiance=10.0)
    shapes.append(carrier)
    light["shape"] = len(shapes) - 1
    points, facets = icosphere(subdivisions)
    shapes.append({"type": "mesh", "objects": [{
        "points": points, "facets": facets,
        "matrix": transform_matrix(n, 0.4, [0.0, -0.6, 0.1]),
        "metalness": 0.0, "roughness": 0.3, "color": [0.8, 0.8, 0.8], "alpha": 1.0}]})
    return {"n": n, "shapes": shapes, "lights": [light],
            "projector": camera(n, 3.0, size), "background": [0.0, 0.0, 0.0]}


def cornell_4d(size=(64, 64, 64), points: int = 20000, seed: int = 2) -> dict:
    """4-space Cornell box: seven 3-parallelotope sides of the 4-cube of edge
    2 (albedo 0.5-0.8), a 3-parallelotope ceiling light of radiance 20, a
    4-parallelotope of edge 0.5 rotated by a seeded SO(4) element, and a
    3-sphere given as the convex hull of `points` points on S^3 (about
    6.7 facets per point), GGX roughness 0.2."""
    n = 4
    colors = {"default": (0.7, 0.7, 0.7),
              (0, -1): (0.8, 0.25, 0.25), (0, 1): (0.25, 0.8, 0.25),
              (1, -1): (0.6, 0.6, 0.6), (1, 1): (0.6, 0.6, 0.6),
              (2, -1): (0.5, 0.5, 0.8), (2, 1): (0.8, 0.8, 0.5),
              (3, 1): (0.7, 0.7, 0.7)}
    shapes = box_walls(n, 1.0, colors, open_axis=n - 1, open_side=-1)
    carrier, light = ceiling_light(n, 1.0, 0.5, up_axis=1, radiance=20.0)
    shapes.append(carrier)
    light["shape"] = len(shapes) - 1
    rot = random_rotation(n, seed)
    edge = 0.5
    center = np.array([0.45, -0.55, 0.35, 0.25])
    vectors = (rot * edge).T
    org = center - 0.5 * vectors.sum(axis=0)
    shapes.append({"type": "parallelotope", "metalness": 0.0, "roughness": 0.2,
                   "color": [0.8, 0.5, 0.3], "alpha": 1.0,
                   "org": org.tolist(), "vectors": vectors.tolist()})
    p, f = convex_hull_mesh(sphere_points(n, points, seed))
    shapes.append({"type": "mesh", "objects": [{
        "points": p, "facets": f,
        "matrix": transform_matrix(n, 0.4, [-0.35, -0.55, -0.25, 0.15]),
        "metalness": 0.0, "roughness": 0.2, "color": [0.75, 0.75, 0.75], "alpha": 1.0}]})
    return {"n": n, "shapes": shapes, "lights": [light],
            "projector": camera(n, 3.0, size), "background": [0.0, 0.0, 0.0]}


def sphere_4d(size=(96, 96, 96), points: int = 150000, seed: int = 3, buckets: int = 64) -> dict:
    """4-space large mesh: the convex hull of `points` points on S^3 with
    radial Gaussian noise (sigma 0.002), lit by one 3-ball light of radius 0.3
    and radiance 30, seen through a parallel projection.  Roughness is uniform
    in [0.1, 0.6] per facet, quantised to `buckets` levels: the reference keeps
    roughness per mesh object (src/painter/shapes/mesh/data.cpp:148-160), so
    each level is one mesh object."""
    n = 4
    p, f = convex_hull_mesh(sphere_points(n, points, seed, noise=0.002))
    rng = np.random.default_rng(seed + 1000)
    roughness = rng.uniform(0.1, 0.6, size=len(f))
    level = np.minimum((roughness - 0.1) / 0.5 * buckets, buckets - 1).astype(np.int64)
    objects = []
    for k in range(buckets):
        sel = f[level == k]
        if len(sel) == 0:
            continue
        objects.append({"points": p, "facets": sel,
                        "matrix": transform_matrix(n, 1.0, [0, 0, 0, 0]),
                        "metalness": 0.0, "roughness": 0.1 + (k + 0.5) * 0.5 / buckets,
                        "color": [0.8, 0.6, 0.4], "alpha": 1.0})
    shapes = [{"type": "mesh", "objects": objects}]
    d = np.array([0.0, -1.0, 0.0, 0.6])
    d /= np.linalg.norm(d)
    light = {"type": "ball", "center": [0.0, 1.7, 0.0, -1.0], "direction": d.tolist(),
             "radius": 0.3, "radiance": [30.0, 30.0, 30.0]}
    org = [0.0, 0.0, 0.0, -3.0]
    units = 2.4 / size[0]
    projector = {"type": "parallel", "org": org, "dir": _unit(n, n - 1),
                 "axes": [_unit(n, k) for k in range(n - 1)], "units_per_pixel": units,
                 "size": list(size)}
    return {"n": n, "shapes": shapes, "lights": [light], "projector": projector,
            "background": [0.0, 0.0, 0.0]}


def cornell_5d(size=(16, 16, 16, 16), points: int = 2000, seed: int = 4) -> dict:
    """5-space box with a ceiling light and a hull mesh of `points` points on
    S^4 (a member of the mixed-scene batch)."""
    n = 5
    colors = {"default": (0.7, 0.7, 0.7), (0, -1): (0.7, 0.1, 0.1), (0, 1): (0.1, 0.7, 0.1)}
    shapes = box_walls(n, 1.0, colors, open_axis=n - 1, open_side=-1)
    carrier, light = ceiling_light(n, 1.0, 0.5, up_axis=1, radiance=30.0)
    shapes.append(carrier)
    light["shape"] = len(shapes) - 1
    p, f = convex_hull_mesh(sphere_points(n, points, seed))
    shapes.append({"type": "mesh", "objects": [{
        "points": p, "facets": f, "matrix": transform_matrix(n, 0.4, [0.0, -0.55, 0.0, 0.1, 0.1]),
        "metalness": 0.0, "roughness": 0.3, "color": [0.8, 0.8, 0.8], "alpha": 1.0}]})
    return {"n": n, "shapes": shapes, "lights": [light],
            "projector": camera(n, 3.0, size), "background": [0.0, 0.0, 0.0]}


def mixed_scene(n: int, points: int, size, seed: int) -> dict:
    """A member of the mixed-scene batch: a box of parallelotope walls open
    on one side, one parallelotope ceiling light, and the convex-hull simplex
    mesh of `points` points on the unit (n-1)-sphere, RGB."""
    rng = np.random.default_rng(seed)
    colors = {"default": (0.7, 0.7, 0.7), (0, -1): (0.75, 0.15, 0.15), (0, 1): (0.15, 0.75, 0.15)}
    shapes = box_walls(n, 1.0, colors, open_axis=n - 1, open_side=-1)
    carrier, light = ceiling_light(n, 1.0, 0.5, up_axis=1, radiance=float(10 * 2 ** (n - 3)))
    shapes.append(carrier)
    light["shape"] = len(shapes) - 1
    p, f = convex_hull_mesh(sphere_points(n, points, seed))
    center = [0.0] * n
    center[1] = -0.55
    shapes.append({"type": "mesh", "objects": [{
        "points": p, "facets": f, "matrix": transform_matrix(n, 0.4, center),
        "metalness": 0.0, "roughness": float(rng.uniform(0.2, 0.6)),
        "color": [0.8, 0.8, 0.8], "alpha": 1.0}]})
    return {"n": n, "shapes": shapes, "lights": [light],
            "projector": camera(n, 3.0, list(size)), "background": [0.0, 0.0, 0.0]}


# screen edge ranges and the largest hull per dimension of the mixed batch
MIXED_SCREENS = {3: (128, 512), 4: (32, 96), 5: (16, 32)}
MIXED_POINTS = {3: (2000, 200000), 4: (2000, 200000), 5: (2000, 50000)}


def _mixed_scene_args(a):
    return mixed_scene(*a)


def stratified_spp(spp: int, dimension: int) -> int:
    """Samples per pixel the stratified jittered sampler renders: spp rounded
    up to k^dimension (src/sampling/sj_sampler.h:51-75)."""
    v = spp ** (1.0 / dimension)
    k = int(math.floor(v))
    if k ** dimension < spp:
        k = int(math.ceil(v))
    return k ** dimension


def _mixed_params(count, seed, points_scale, screen_scale, spp, depth):
    """((n, points, screen, hull seed), spp, depth, points) of each job of the batch."""
    rng = np.random.default_rng(seed)
    params = []
    for k in range(count):
        n = int(rng.integers(3, 6))
        lo, hi = MIXED_POINTS[n]
        points = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi))) * points_scale))
        points = max(points, 4 * n)
        a, b = MIXED_SCREENS[n]
        edge = max(4, int(round(rng.uniform(a, b) * screen_scale)))
        job_spp = int(round(math.exp(rng.uniform(math.log(spp[0]), math.log(spp[1])))))
        job_depth = int(rng.integers(depth[0], depth[1] + 1))
        params.append(((n, points, [edge] * (n - 1), seed * 1000 + k), job_spp, job_depth, points))
    return params


def mixed_batch_hulls(count: int = 64, seed: int = 4, points_scale: float = 1.0) -> list[tuple[int, int, int, int]]:
    """(job index, dimension, points, point seed) of every job's hull in the
    mixed batch, without building it: the hull is of
    sphere_points(dimension, points, point seed)."""
    params = _mixed_params(count, seed, points_scale, 1.0, (4, 64), (5, 8))
    return [(k, p[0][0], p[0][1], p[0][3]) for k, p in enumerate(params)]


def mixed_batch(count: int = 64, seed: int = 4, points_scale: float = 1.0, screen_scale: float = 1.0,
                spp=(4, 64), depth=(5, 8), workers: int = 1, select=None) -> list[dict]:
    """Jobs of the batched mixed-scene workload: dimension uniform in
    {3, 4, 5}; hull of N points on the unit sphere with N log-uniform in the
    dimension's range (MIXED_POINTS: 2k-200k, at most 50k in 5-space, where
    hulls grow fastest); screen edge uniform in MIXED_SCREENS; samples per
    pixel log-uniform in `spp`; maximum depth uniform in `depth`.  The scale
    arguments shrink hulls and screens for quick runs.  With `workers` > 1
    the hulls are computed in that many processes (started with `spawn`, so
    a process that already uses the GPU can call it); the jobs are the same.
    `select`: indices of the jobs to build (the others are left out); every
    job carries "paths", its paths per pass."""
    params = _mixed_params(count, seed, points_scale, screen_scale, spp, depth)
    chosen = list(range(count)) if select is None else sorted(set(select))
    params = [params[i] for i in chosen]
    count = len(params)
    args = [p[0] for p in params]
    if workers > 1 and count > 1:
        import multiprocessing

        # largest hulls first, so the pool's last tasks are short
        order = sorted(range(count), key=lambda i: -(args[i][1] * 4 ** args[i][0]))
        with multiprocessing.get_context("spawn").Pool(min(workers, count)) as pool:
            built = pool.map(_mixed_scene_args, [args[i] for i in order], chunksize=1)
        descs = [None] * count
        for i, d in zip(order, built):
            descs[i] = d
    else:
        descs = [mixed_scene(*a) for a in args]
    return [{"desc": d, "spp": p[1], "max_depth": p[2], "points": p[3], "index": i,
             "paths": int(np.prod(p[0][2])) * stratified_spp(p[1], p[0][0] - 1)}
            for i, d, p in zip(chosen, descs, params)]


def mixed_batch_paths(count: int = 64, seed: int = 4, screen_scale: float = 1.0, spp=(4, 64)) -> list[int]:
    """Paths per pass of each job of mixed_batch, without building scenes."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.integers(3, 6))
        rng.uniform()  # hull points
        a, b = MIXED_SCREENS[n]
        edge = max(4, int(round(rng.uniform(a, b) * screen_scale)))
        job_spp = int(round(math.exp(rng.uniform(math.log(spp[0]), math.log(spp[1])))))
        rng.integers(5, 9)  # depth
        out.append(edge ** (n - 1) * stratified_spp(job_spp, n - 1))
    return out


CONFIGS = {
    "cornell3d": cornell_3d,
    "cornell4d": cornell_4d,
    "sphere4d": sphere_4d,
    "cornell5d": cornell_5d,
}


def describe(scene: dict) -> dict:
    """Counts of a scene description (for logs and bench config lines)."""
    facets = sum(len(o["facets"]) for s in scene["shapes"] if s["type"] == "mesh" for o in s["objects"])
    return {"n": scene["n"], "shapes": len(scene["shapes"]), "lights": len(scene["lights"]),
            "facets": int(facets), "screen": list(scene["projector"]["size"])}
