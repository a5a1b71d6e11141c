"""Generates the golden fixtures in this directory from the CPU oracle
(the reference painter compiled from its own sources, oracle/_ref).

    python tests/golden/make_golden.py

Fixtures (numpy .npz):
  rng.npz      PCG32 draws, uniform [0, 1) draws and stratified jittered
               points of seed_seq streams, float and double
  cornell3d.npz  3-space Cornell box (16x16, icosphere of 1,280 triangles),
               double precision, RGB: the painter's mesh data, per-sample
               BPT colours of one seeded pass (16 spp, depth 5), the
               reference's filtered trimmed image, and closest-hit facet
               indices and distances of a seeded ray set
  cornell4d.npz  4-space Cornell box (6x6x6, hull of 600 points on S^3),
               double precision, 64-bin spectrum, 8 spp, depth 6
  cornell5d.npz  5-space box (4x4x4x4, hull of 200 points on S^4), double,
               RGB, 16 spp, depth 5
  pt.npz       the PT integrator (src/painter/integrators/pt/pt.cpp) on the
               three boxes above (keys <name>_colors, _valid, _rgb, _rgba;
               same scenes, seeds and sample points) and on a 4-space sphere
               lit by a ball light (8x8x8, hull of 2,000 points, RGB, 16 spp;
               keys sphere4d_*, with its mesh arrays)

    python tests/golden/make_golden.py pt    # pt.npz only
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from math_b200 import scenes  # noqa: E402
from oracle import oracle  # noqa: E402

OUT = Path(__file__).resolve().parent

SEEDS = [[1, 2, 3, 4], [7], [123456789, 42], [0, 0, 0, 1]]


def rng_fixture():
    out = {}
    for i, w in enumerate(SEEDS):
        out[f"seed_{i}"] = np.asarray(w, np.uint32)
        out[f"pcg_{i}"] = oracle.pcg(w, 64)
        out[f"canonical_double_{i}"] = oracle.canonical(w, 64, True)
        out[f"canonical_float_{i}"] = oracle.canonical(w, 64, False)
        for dim in (2, 3, 4):
            for dbl in (True, False):
                out[f"sj_{dim}_{int(dbl)}_{i}"] = oracle.sj_points(dim, 16 if dim < 4 else 81, w, dbl)
    np.savez_compressed(OUT / "rng.npz", **out)


def mesh_arrays(scene: oracle.Scene) -> dict:
    m = scene.mesh_dump()
    return {"vertices": m["vertices"], "normals": m["normals"], "facets": m["facets"],
            "facet_material": m["facet_material"], "material_params": m["material_params"],
            "material_colors": m["material_colors"], "planes": m["planes"],
            "node_bounds": m["node_bounds"], "node_info": m["node_info"], "indices": m["indices"]}


def seeded_rays(n: int, count: int, seed: int, half: float) -> np.ndarray:
    rng = np.random.default_rng(seed)
    org = rng.uniform(-half, half, size=(count, n))
    d = rng.normal(size=(count, n))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([org, d], axis=1)


def scene_fixture(name: str, desc: dict, spectrum: bool, spp: int, depth: int, rays: int):
    s = oracle.Scene(desc, "double", spectrum)
    out = {f"mesh_{k}": v for k, v in mesh_arrays(s).items()}
    if desc["n"] == 5:
        # the facet and BVH records are checked on the smaller fixtures
        for k in ("planes", "node_bounds", "node_info", "indices"):
            del out[f"mesh_{k}"]
    points, colors, valid = s.render_samples(spp, depth, seed=1, pass_index=0)
    out.update(points=points, colors=colors, valid=valid, spp=np.int32(spp), depth=np.int32(depth))
    rgb, rgba = s.render_image(spp, depth, seed=1, passes=1)
    out.update(rgb=rgb, rgba=rgba)
    r = seeded_rays(desc["n"], rays, 11, 1.2)
    facet, t = s.mesh_trace(r)
    hit, st, sp, sn = s.scene_trace(r)
    out.update(rays=r, ray_facet=facet, ray_t=t, scene_hit=hit, scene_t=st, scene_point=sp)
    np.savez_compressed(OUT / f"{name}.npz", **out)


def small_scenes() -> dict:
    return {
        "cornell3d": (scenes.cornell_3d(size=(16, 16), subdivisions=3), False, 16, 5),
        "cornell4d": (scenes.cornell_4d(size=(6, 6, 6), points=600), True, 8, 6),
        "cornell5d": (scenes.cornell_5d(size=(4, 4, 4, 4), points=200), False, 16, 5),
    }


def pt_sphere_scene() -> tuple:
    return scenes.sphere_4d(size=(8, 8, 8), points=2000, buckets=4), False, 16


def pt_fixture():
    out = {}

    def render(prefix: str, s: oracle.Scene, spp: int, depth: int):
        s.set_integrator("pt")
        _, colors, valid = s.render_samples(spp, depth, seed=1, pass_index=0)
        rgb, rgba = s.render_image(spp, depth, seed=1, passes=1)
        out.update({f"{prefix}_colors": colors, f"{prefix}_valid": valid, f"{prefix}_rgb": rgb,
                    f"{prefix}_rgba": rgba})

    for name, (desc, spectrum, spp, depth) in small_scenes().items():
        render(name, oracle.Scene(desc, "double", spectrum), spp, depth)
    desc, spectrum, spp = pt_sphere_scene()
    s = oracle.Scene(desc, "double", spectrum)
    out.update({f"sphere4d_mesh_{k}": v for k, v in mesh_arrays(s).items()
                if k not in ("planes", "node_bounds", "node_info", "indices")})
    out["sphere4d_spp"] = np.int32(spp)
    render("sphere4d", s, spp, 1)
    np.savez_compressed(OUT / "pt.npz", **out)


def main():
    if sys.argv[1:] == ["pt"]:
        pt_fixture()
        return
    rng_fixture()
    for name, (desc, spectrum, spp, depth) in small_scenes().items():
        scene_fixture(name, desc, spectrum, spp, depth, rays=4096)
    pt_fixture()


if __name__ == "__main__":
    main()
