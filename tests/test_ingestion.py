"""Mesh ingestion on the host, no GPU: the library's mesh data (used points
renumbered by first use, vertex normals, the object's transform, facets)
against the reference's (src/painter/shapes/mesh/data.cpp:88-200 over
src/model/mesh/create_facets.cpp and normals.cpp) read from the oracle.
Everything is compared bit for bit, the normals' signs included: the sign
of a vertex normal decides which way a facet's geometric normal faces
(src/painter/shapes/mesh/facet.cpp:104-117)."""

from __future__ import annotations

import numpy as np
import pytest

from math_b200 import painter as P
from math_b200 import scenes


def ingest(desc: dict, precision: str = "double") -> dict:
    """Adds the scene's first mesh shape to a library scene that is never
    finalized, and reads back the ingested mesh."""
    L = P.lib()
    n = desc["n"]
    h = L.nbpt_scene_create(n, 1 if precision == "double" else 0, 0)
    assert h, L.nbpt_last_error()
    try:
        mesh = next(s for s in desc["shapes"] if s["type"] == "mesh")
        for o in mesh["objects"]:
            pts = P._f(o["points"]).reshape(-1, n)
            fac = P._i(o["facets"]).reshape(-1, n)
            P._check(L.nbpt_scene_add_mesh_object(
                h, P._p(pts, P._F), len(pts), P._p(fac, P._I), len(fac),
                P._p(P._d(o["matrix"]).reshape(-1), P._D), P._null(P._F), o["metalness"], o["roughness"],
                P._p(P._f(o["color"]), P._F), o["alpha"]))
        P._check(L.nbpt_scene_add_mesh(h))
        counts = np.zeros(3, np.int64)
        P._check(L.nbpt_scene_ingested_mesh(h, 0, P._p(counts, P._L), None, None, None))
        v = np.zeros((counts[0], n))
        nn = np.zeros((counts[2], n))
        f = np.zeros((counts[1], n), np.int32)
        P._check(L.nbpt_scene_ingested_mesh(h, 0, P._p(counts, P._L), P._p(v, P._D), P._p(nn, P._D),
                                           P._p(f, P._I)))
        return {"vertices": v, "normals": nn, "facets": f}
    finally:
        L.nbpt_scene_destroy(h)


def rotated(desc: dict, seed: int) -> dict:
    """The scene with its mesh turned by a seeded rotation and scaled
    unevenly, so the normals go through a full inverse transpose."""
    n = desc["n"]
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.normal(size=(n, n)))
    m = np.eye(n + 1)
    m[:n, :n] = q @ np.diag(rng.uniform(0.3, 0.5, n))
    m[:n, n] = rng.uniform(-0.2, 0.2, n)
    for s in desc["shapes"]:
        if s["type"] == "mesh":
            for o in s["objects"]:
                o["matrix"] = m.tolist()
    return desc


CASES = {
    "3-space icosphere": lambda: scenes.cornell_3d(size=(4, 4), subdivisions=3),
    "4-space hull": lambda: scenes.cornell_4d(size=(4, 4, 4), points=3000),
    "5-space hull": lambda: scenes.cornell_5d(size=(4, 4, 4, 4), points=600),
    "3-space rotated": lambda: rotated(scenes.cornell_3d(size=(4, 4), subdivisions=2), 5),
    "4-space rotated": lambda: rotated(scenes.cornell_4d(size=(4, 4, 4), points=1000), 6),
    "5-space rotated": lambda: rotated(scenes.cornell_5d(size=(4, 4, 4, 4), points=400), 7),
    "4-space, 8 objects sharing points": lambda: scenes.sphere_4d(size=(4, 4, 4), points=800, buckets=8),
}


@pytest.mark.parametrize("case", list(CASES))
def test_ingested_mesh_equals_the_reference(oracle_lib, case):
    desc = CASES[case]()
    ours = ingest(desc)
    ref = oracle_lib.Scene(desc, "double", False).mesh_dump()
    assert np.array_equal(ours["facets"], ref["facets"])
    assert np.array_equal(ours["vertices"], ref["vertices"])
    assert np.array_equal(ours["normals"], ref["normals"])


def test_ingested_mesh_needs_no_device():
    desc = scenes.cornell_3d(size=(4, 4), subdivisions=1)
    m = ingest(desc)
    assert m["vertices"].shape == (42, 3) and m["normals"].shape == (42, 3)
    assert m["facets"].shape == (80, 3)
    assert np.allclose(np.linalg.norm(m["normals"], axis=1), 2.5, rtol=1e-6)  # unit normals / scale 0.4
