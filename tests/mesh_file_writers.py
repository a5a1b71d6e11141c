"""Writers of n-dimensional OBJ and STL files for the mesh-file tests, in the
layouts the reference's loaders read (src/model/mesh/file/load_obj.cpp,
load_stl.cpp): OBJ "v", "vn", "f v//n" lines with "usemtl" / "mtllib" and a
.mtl of "newmtl" / "Kd"; STL ASCII ("solid" ... "endsolid") and binary (an
80-byte header, a uint32 facet count, then per facet N normal floats and N
vertices of N floats)."""

from __future__ import annotations

import struct
from pathlib import Path

import numpy as np


def obj_extension(n: int) -> str:
    return ".obj" if n == 3 else f".obj{n}"


def stl_extension(n: int) -> str:
    return ".stl" if n == 3 else f".stl{n}"


def facet_normals(points: np.ndarray, facets: np.ndarray) -> np.ndarray:
    """Unit normals of the facets (any orientation), for the STL normal field."""
    n = points.shape[1]
    out = np.zeros((len(facets), n))
    for i, f in enumerate(facets):
        e = points[f[1:]] - points[f[0]]
        # the null space of the edge vectors
        _, _, vt = np.linalg.svd(e)
        out[i] = vt[-1]
    return out


def write_obj(path: Path, points, facets, normals=None, with_normals=None, materials=None, facet_material=None,
              relative_every: int = 0):
    """points [V, n], facets [F, n]; normals [V, n] used as "vn" for the
    facets where with_normals is true; materials: {name: (r, g, b)} written to
    a .mtl beside the file, facet_material: the name per facet (None: none);
    every `relative_every`-th facet uses negative (relative) indices."""
    path = Path(path)
    points = np.asarray(points)
    facets = np.asarray(facets)
    n = points.shape[1]
    lines = ["# n-dimensional OBJ written by the tests"]
    if materials:
        lib = path.with_suffix(".mtl").name
        lines.append(f"mtllib {lib}")
        with open(path.parent / lib, "w") as f:
            for name, rgb in materials.items():
                f.write(f"newmtl {name}\nKd {rgb[0]:.6f} {rgb[1]:.6f} {rgb[2]:.6f}\n\n")
    for p in points:
        lines.append("v " + " ".join(repr(float(np.float32(x))) for x in p))
    if normals is not None:
        for v in normals:
            lines.append("vn " + " ".join(repr(float(np.float32(x))) for x in v))
    current = None
    for i, f in enumerate(facets):
        name = facet_material[i] if facet_material is not None else None
        if name is not None and name != current:
            lines.append(f"usemtl {name}")
            current = name
        has_n = normals is not None and (with_normals is None or with_normals[i])
        relative = relative_every > 0 and i % relative_every == 0
        corners = []
        for v in f:
            vi = int(v) - len(points) if relative else int(v) + 1
            if has_n:
                ni = int(v) - len(points) if relative else int(v) + 1
                corners.append(f"{vi}//{ni}")
            else:
                corners.append(f"{vi}")
        lines.append("f " + " ".join(corners) + ("  # facet" if i % 7 == 3 else ""))
    path.write_text("\n".join(lines) + "\n")


def write_stl_ascii(path: Path, points, facets):
    points = np.asarray(points, np.float32)
    facets = np.asarray(facets)
    normals = facet_normals(points.astype(np.float64), facets).astype(np.float32)
    out = ["solid tests"]
    for f, nrm in zip(facets, normals):
        out.append(" facet normal " + " ".join(repr(float(x)) for x in nrm))
        out.append("  outer loop")
        for v in f:
            out.append("   vertex " + " ".join(repr(float(x)) for x in points[v]))
        out.append("  endloop")
        out.append(" endfacet")
    out.append("endsolid tests")
    Path(path).write_text("\n".join(out) + "\n")


def write_stl_binary(path: Path, points, facets):
    points = np.asarray(points, np.float32)
    facets = np.asarray(facets)
    normals = facet_normals(points.astype(np.float64), facets).astype(np.float32)
    with open(path, "wb") as f:
        f.write(b"binary n-dimensional STL written by the tests".ljust(80, b" "))
        f.write(struct.pack("<I", len(facets)))
        for fa, nrm in zip(facets, normals):
            f.write(nrm.tobytes())
            f.write(points[fa].tobytes())
