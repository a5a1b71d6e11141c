"""ctypes binding of the CPU test oracle (oracle/_ref/libnbpt_oracle.so).

Test infrastructure only: the tests, the golden-fixture generator and the
CPU-baseline leg of bench.py use it as the checker.  The library is the
reference painter compiled from its own sources (oracle/Makefile) plus the
project-written driver (oracle/driver.cpp); scenes are built through the
reference's own constructors from the same scene descriptions
(math_b200/scenes.py) the accelerated library consumes.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_ref" / "libnbpt_oracle.so"

_lib = None

_P = ctypes.c_void_p
_D = ctypes.POINTER(ctypes.c_double)
_F = ctypes.POINTER(ctypes.c_float)
_I = ctypes.POINTER(ctypes.c_int)
_U = ctypes.POINTER(ctypes.c_uint)
_B = ctypes.POINTER(ctypes.c_ubyte)
_L = ctypes.POINTER(ctypes.c_longlong)


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"oracle library not built: {LIB_PATH} (run make -C oracle)")
        L = ctypes.CDLL(str(LIB_PATH))
        sig = {
            "oracle_last_error": (ctypes.c_char_p, []),
            "oracle_scene_new": (_P, [ctypes.c_int, ctypes.c_int, ctypes.c_int]),
            "oracle_scene_free": (None, [_P]),
            "oracle_scene_add_hyperplane_parallelotope": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, _F, ctypes.c_double, _D, _D]),
            "oracle_scene_add_parallelotope": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, _F, ctypes.c_double, _D, _D]),
            "oracle_scene_add_mesh_object": (ctypes.c_int, [_P, _F, ctypes.c_long, _I, ctypes.c_long, _D, ctypes.c_double, ctypes.c_double, _F, ctypes.c_double]),
            "oracle_scene_add_mesh": (ctypes.c_int, [_P]),
            "oracle_scene_add_mesh_file": (ctypes.c_int, [_P, ctypes.c_char_p, _D, ctypes.c_double, ctypes.c_double, _F, ctypes.c_double]),
            "oracle_load_mesh_file": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _L]),
            "oracle_mesh_file_arrays": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _L, _F, _F, _I, _I, _B, _I]),
            "oracle_scene_add_parallelotope_light": (ctypes.c_int, [_P, ctypes.c_int, _D, _F]),
            "oracle_scene_add_ball_light": (ctypes.c_int, [_P, _D, _D, ctypes.c_double, _F]),
            "oracle_scene_set_perspective": (ctypes.c_int, [_P, _D, _D, _D, ctypes.c_double, _I]),
            "oracle_scene_set_parallel": (ctypes.c_int, [_P, _D, _D, _D, ctypes.c_double, _I]),
            "oracle_scene_finalize": (ctypes.c_int, [_P, _F]),
            "oracle_scene_pixel_count": (ctypes.c_longlong, [_P]),
            "oracle_scene_actual_spp": (ctypes.c_int, [_P, ctypes.c_int]),
            "oracle_scene_set_integrator": (ctypes.c_int, [_P, ctypes.c_int]),
            "oracle_scene_set_flat_shading": (ctypes.c_int, [_P, ctypes.c_int]),
            "oracle_render_samples": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, ctypes.c_uint, ctypes.c_uint, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_int, _D, _F, _B]),
            "oracle_render_image": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, ctypes.c_uint, ctypes.c_int, ctypes.c_int, _F, _F]),
            "oracle_render_image_range": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, ctypes.c_uint, ctypes.c_int, ctypes.c_int, ctypes.c_longlong, ctypes.c_longlong, _F, _F]),
            "oracle_paint": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D, _F]),
            "oracle_mesh_info": (ctypes.c_int, [_P, ctypes.c_int, _L]),
            "oracle_mesh_dump": (ctypes.c_int, [_P, ctypes.c_int, _D, _D, _I, _I, _D, _F, _D, _D, _U, _U]),
            "oracle_mesh_trace": (ctypes.c_int, [_P, ctypes.c_int, _D, ctypes.c_longlong, ctypes.c_double, ctypes.c_int, _I, _D, _B, ctypes.c_int]),
            "oracle_scene_trace": (ctypes.c_int, [_P, _D, ctypes.c_longlong, ctypes.c_int, _D, _D, _D, _B]),
            "oracle_brdf": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, _F, _D, _D, _D, _F, _D]),
            "oracle_brdf_sample": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, _F, _D, _D, _U, ctypes.c_int, _D, _D, _F]),
            "oracle_light_sample": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, _U, ctypes.c_int, _D, _D, _D, _F]),
            "oracle_pcg": (ctypes.c_int, [_U, ctypes.c_int, ctypes.c_int, _U]),
            "oracle_canonical": (ctypes.c_int, [_U, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D]),
            "oracle_sj_points": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _U, ctypes.c_int, _D]),
            "oracle_f1_albedo_tables": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _F, _F]),
            "oracle_f1_albedo_tables_double": (ctypes.c_int, [ctypes.c_int, _D, _D]),
            "oracle_spectrum_functions": (ctypes.c_int, [_D]),
            "oracle_color": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _F, _F]),
            "oracle_constants": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _D]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class OracleError(RuntimeError):
    pass


def _check(r):
    if r is None or (isinstance(r, int) and r < 0):
        raise OracleError(lib().oracle_last_error().decode())
    return r


def _d(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _f(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _i(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def _seed(words) -> tuple[np.ndarray, int]:
    w = np.ascontiguousarray(np.asarray(words, dtype=np.uint32))
    return w, len(w)


def channels(spectrum: bool) -> int:
    return 64 if spectrum else 3


class Scene:
    """A reference-painter scene built from a scene description."""

    def __init__(self, desc: dict, precision: str = "double", spectrum: bool = False):
        L = lib()
        self.n = desc["n"]
        self.spectrum = spectrum
        self.channels = channels(spectrum)
        self.h = L.oracle_scene_new(self.n, 1 if precision == "double" else 0, 1 if spectrum else 0)
        if not self.h:
            raise OracleError(L.oracle_last_error().decode())
        self.mesh_shapes = []
        n = self.n
        for s in desc["shapes"]:
            kind = s["type"]
            if kind == "hyperplane_parallelotope":
                _check(L.oracle_scene_add_hyperplane_parallelotope(
                    self.h, s["metalness"], s["roughness"], ptr(_f(s["color"]), _F), s["alpha"],
                    ptr(_d(s["org"]), _D), ptr(_d(s["vectors"]).reshape(-1), _D)))
            elif kind == "parallelotope":
                _check(L.oracle_scene_add_parallelotope(
                    self.h, s["metalness"], s["roughness"], ptr(_f(s["color"]), _F), s["alpha"],
                    ptr(_d(s["org"]), _D), ptr(_d(s["vectors"]).reshape(-1), _D)))
            elif kind == "mesh":
                for o in s["objects"]:
                    if "file" in o:
                        _check(L.oracle_scene_add_mesh_file(
                            self.h, str(o["file"]).encode(), ptr(_d(o["matrix"]).reshape(-1), _D),
                            o["metalness"], o["roughness"], ptr(_f(o["color"]), _F), o["alpha"]))
                        continue
                    pts = _f(o["points"]).reshape(-1, n)
                    fac = _i(o["facets"]).reshape(-1, n)
                    _check(L.oracle_scene_add_mesh_object(
                        self.h, ptr(pts, _F), len(pts), ptr(fac, _I), len(fac),
                        ptr(_d(o["matrix"]).reshape(-1), _D), o["metalness"], o["roughness"],
                        ptr(_f(o["color"]), _F), o["alpha"]))
                self.mesh_shapes.append(_check(L.oracle_scene_add_mesh(self.h)))
            else:
                raise ValueError(f"unknown shape type {kind}")
        for l in desc["lights"]:
            if l["type"] == "parallelotope":
                _check(L.oracle_scene_add_parallelotope_light(
                    self.h, l["shape"], ptr(_d(l["direction"]), _D), ptr(_f(l["radiance"]), _F)))
            elif l["type"] == "ball":
                _check(L.oracle_scene_add_ball_light(
                    self.h, ptr(_d(l["center"]), _D), ptr(_d(l["direction"]), _D), l["radius"],
                    ptr(_f(l["radiance"]), _F)))
            else:
                raise ValueError(f"unknown light type {l['type']}")
        p = desc["projector"]
        size = _i(p["size"])
        if p["type"] == "perspective":
            _check(L.oracle_scene_set_perspective(
                self.h, ptr(_d(p["org"]), _D), ptr(_d(p["dir"]), _D),
                ptr(_d(p["axes"]).reshape(-1), _D), p["fov"], ptr(size, _I)))
        else:
            _check(L.oracle_scene_set_parallel(
                self.h, ptr(_d(p["org"]), _D), ptr(_d(p["dir"]), _D),
                ptr(_d(p["axes"]).reshape(-1), _D), p["units_per_pixel"], ptr(size, _I)))
        _check(L.oracle_scene_finalize(self.h, ptr(_f(desc["background"]), _F)))
        self.size = [int(x) for x in p["size"]]
        self.pixels = int(np.prod(self.size))

    def __del__(self):
        h = getattr(self, "h", None)
        if h and _lib is not None:
            _lib.oracle_scene_free(h)
            self.h = None

    def actual_spp(self, spp: int) -> int:
        return _check(lib().oracle_scene_actual_spp(self.h, spp))

    def set_flat_shading(self, flat: bool):
        """create_painter's flat_shading for render_samples, render_image and paint."""
        _check(lib().oracle_scene_set_flat_shading(self.h, 1 if flat else 0))

    def set_integrator(self, integrator: str):
        """'bpt' (the default) or 'pt' for render_samples, render_image and paint."""
        if integrator not in ("bpt", "pt"):
            raise ValueError(f"Unknown integrator {integrator!r}")
        _check(lib().oracle_scene_set_integrator(self.h, {"bpt": 0, "pt": 1}[integrator]))

    def render_samples(self, spp: int, max_depth: int, seed: int, pass_index: int = 0,
                       begin: int = 0, end: int | None = None, threads: int | None = None):
        """Per-sample output of one seeded pass over pixels [begin, end):
        (points [P, S, n-1] float64, colors [P, S, C] float32, valid [P, S] bool)."""
        end = self.pixels if end is None else end
        s = self.actual_spp(spp)
        count = end - begin
        points = np.zeros((count, s, self.n - 1), np.float64)
        colors = np.zeros((count, s, self.channels), np.float32)
        valid = np.zeros((count, s), np.uint8)
        _check(lib().oracle_render_samples(
            self.h, spp, max_depth, seed, pass_index, begin, end, threads or os.cpu_count(),
            ptr(points, _D), ptr(colors, _F), ptr(valid, _B)))
        return points, colors, valid.astype(bool)

    def render_image(self, spp: int, max_depth: int, seed: int, passes: int = 1, threads: int | None = None):
        """Seeded passes accumulated by the reference's pixels::Pixels:
        (rgb [P, 3], rgba [P, 4]) float32."""
        rgb = np.zeros((self.pixels, 3), np.float32)
        rgba = np.zeros((self.pixels, 4), np.float32)
        _check(lib().oracle_render_image(self.h, spp, max_depth, seed, passes, threads or os.cpu_count(),
                                         ptr(rgb, _F), ptr(rgba, _F)))
        return rgb, rgba

    def render_image_range(self, spp: int, max_depth: int, seed: int, begin: int, end: int, passes: int = 1,
                           threads: int | None = None):
        """render_image from the samples of pixels [begin, end) only: pixels
        whose every source lies in the range are complete."""
        rgb = np.zeros((self.pixels, 3), np.float32)
        rgba = np.zeros((self.pixels, 4), np.float32)
        _check(lib().oracle_render_image_range(self.h, spp, max_depth, seed, passes, threads or os.cpu_count(),
                                               begin, end, ptr(rgb, _F), ptr(rgba, _F)))
        return rgb, rgba

    def paint(self, spp: int, max_depth: int, passes: int = 1, threads: int | None = None):
        """The unmodified reference painter.  Returns (stats dict, rgb [P, 3])."""
        stats = np.zeros(5, np.float64)
        rgb = np.zeros((self.pixels, 3), np.float32)
        _check(lib().oracle_paint(self.h, spp, max_depth, passes, threads or os.cpu_count(),
                                  ptr(stats, _D), ptr(rgb, _F)))
        return {"sample_count": int(stats[0]), "ray_count": int(stats[1]),
                "pass_duration": float(stats[2]), "wall": float(stats[3]),
                "pass_number": int(stats[4])}, rgb

    def mesh_dump(self, shape: int | None = None) -> dict:
        shape = self.mesh_shapes[0] if shape is None else shape
        n, C = self.n, self.channels
        counts = np.zeros(6, np.int64)
        _check(lib().oracle_mesh_info(self.h, shape, ptr(counts, _L)))
        nv, nn, nf, nm, nodes, ni = (int(x) for x in counts)
        out = {
            "vertices": np.zeros((nv, n)), "normals": np.zeros((nn, n)),
            "facets": np.zeros((nf, n), np.int32), "facet_material": np.zeros(nf, np.int32),
            "material_params": np.zeros((nm, 3)), "material_colors": np.zeros((nm, C), np.float32),
            "planes": np.zeros((nf, n, n + 1)), "node_bounds": np.zeros((nodes, 2, n)),
            "node_info": np.zeros((nodes, 3), np.uint32), "indices": np.zeros(ni, np.uint32),
        }
        _check(lib().oracle_mesh_dump(
            self.h, shape, ptr(out["vertices"], _D), ptr(out["normals"], _D), ptr(out["facets"], _I),
            ptr(out["facet_material"], _I), ptr(out["material_params"], _D),
            ptr(out["material_colors"], _F), ptr(out["planes"], _D), ptr(out["node_bounds"], _D),
            ptr(out["node_info"], _U), ptr(out["indices"], _U)))
        return out

    def mesh_trace(self, rays: np.ndarray, any_hit: bool = False, max_distance: float = np.inf,
                   shape: int | None = None, threads: int | None = None):
        """Closest hit (facet index or -1, t) or any hit (bool) against one mesh."""
        shape = self.mesh_shapes[0] if shape is None else shape
        rays = _d(rays).reshape(-1, 2 * self.n)
        m = len(rays)
        facet = np.zeros(m, np.int32)
        t = np.zeros(m)
        anyh = np.zeros(m, np.uint8)
        _check(lib().oracle_mesh_trace(self.h, shape, ptr(rays, _D), m, max_distance, 1 if any_hit else 0,
                                       ptr(facet, _I), ptr(t, _D), ptr(anyh, _B), threads or os.cpu_count()))
        return anyh.astype(bool) if any_hit else (facet, t)

    def scene_trace(self, rays: np.ndarray, threads: int | None = None):
        rays = _d(rays).reshape(-1, 2 * self.n)
        m = len(rays)
        t = np.zeros(m)
        point = np.zeros((m, self.n))
        normal = np.zeros((m, self.n))
        hit = np.zeros(m, np.uint8)
        _check(lib().oracle_scene_trace(self.h, ptr(rays, _D), m, threads or os.cpu_count(), ptr(t, _D),
                                        ptr(point, _D), ptr(normal, _D), ptr(hit, _B)))
        return hit.astype(bool), t, point, normal

    def brdf(self, metalness, roughness, rgb, n, v, l):
        f = np.zeros(self.channels, np.float32)
        pdf = np.zeros(1)
        _check(lib().oracle_brdf(self.h, metalness, roughness, ptr(_f(rgb), _F), ptr(_d(n), _D),
                                 ptr(_d(v), _D), ptr(_d(l), _D), ptr(f, _F), ptr(pdf, _D)))
        return f, float(pdf[0])

    def brdf_sample(self, metalness, roughness, rgb, n, v, seed_words):
        w, k = _seed(seed_words)
        l = np.zeros(self.n)
        pdf = np.zeros(1)
        f = np.zeros(self.channels, np.float32)
        _check(lib().oracle_brdf_sample(self.h, metalness, roughness, ptr(_f(rgb), _F), ptr(_d(n), _D),
                                        ptr(_d(v), _D), ptr(w, _U), k, ptr(l, _D), ptr(pdf, _D), ptr(f, _F)))
        return l, float(pdf[0]), f

    def light_sample(self, light: int, kind: str, seed_words, point=None, normal=None):
        w, k = _seed(seed_words)
        out = np.zeros(3 * self.n + 2)
        rad = np.zeros(self.channels, np.float32)
        point = _d(point if point is not None else np.zeros(self.n))
        normal = _d(normal if normal is not None else np.zeros(self.n))
        _check(lib().oracle_light_sample(self.h, light, 0 if kind == "leave" else 1, ptr(w, _U), k,
                                         ptr(point, _D), ptr(normal, _D), ptr(out, _D), ptr(rad, _F)))
        return out, rad


def pcg(seed_words, count: int) -> np.ndarray:
    w, k = _seed(seed_words)
    out = np.zeros(count, np.uint32)
    _check(lib().oracle_pcg(ptr(w, _U), k, count, ptr(out, _U)))
    return out


def canonical(seed_words, count: int, double: bool = True) -> np.ndarray:
    w, k = _seed(seed_words)
    out = np.zeros(count)
    _check(lib().oracle_canonical(ptr(w, _U), k, count, 1 if double else 0, ptr(out, _D)))
    return out


def sj_points(dimension: int, spp: int, seed_words, double: bool = True) -> np.ndarray:
    w, k = _seed(seed_words)
    count = _check(lib().oracle_sj_points(dimension, 1 if double else 0, spp, ptr(w, _U), k,
                                          ctypes.cast(None, _D)))
    out = np.zeros((count, dimension))
    _check(lib().oracle_sj_points(dimension, 1 if double else 0, spp, ptr(w, _U), k, ptr(out, _D)))
    return out


def f1_albedo_tables(n: int) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
    """(float table [32*32], float average [32], double table, double average)."""
    tf = np.zeros(1024, np.float32)
    af = np.zeros(32, np.float32)
    td = np.zeros(1024)
    ad = np.zeros(32)
    _check(lib().oracle_f1_albedo_tables(n, 0, ptr(tf, _F), ptr(af, _F)))
    _check(lib().oracle_f1_albedo_tables_double(n, ptr(td, _D), ptr(ad, _D)))
    return tf, af, td, ad


def spectrum_functions() -> np.ndarray:
    out = np.zeros((17, 64))
    _check(lib().oracle_spectrum_functions(ptr(out, _D)))
    return out


def color(rgb, spectrum: bool, illuminant: bool) -> np.ndarray:
    out = np.zeros(channels(spectrum), np.float32)
    _check(lib().oracle_color(1 if spectrum else 0, 1 if illuminant else 0, ptr(_f(rgb), _F), ptr(out, _F)))
    return out


def constants(n: int, double: bool) -> np.ndarray:
    out = np.zeros(8)
    _check(lib().oracle_constants(n, 1 if double else 0, ptr(out, _D)))
    return out


def load_mesh_file(path, n: int) -> dict:
    """The reference's own OBJ / STL loader on `path`: counts of the mesh it
    reads (vertices, normals, facets)."""
    counts = np.zeros(3, np.int64)
    stl = 1 if ".stl" in str(path).lower() else 0
    _check(lib().oracle_load_mesh_file(str(path).encode(), n, stl, ptr(counts, _L)))
    return {"vertices": int(counts[0]), "normals": int(counts[1]), "facets": int(counts[2])}


def mesh_file_arrays(path, n: int) -> dict:
    """The mesh the reference's own OBJ / STL loader reads from `path`, as
    arrays: vertices [V, n], normals [M, n], and per facet its vertex and
    normal indices [F, n] (-1 where the facet has no normals), has_normal [F]
    and material [F] (-1: none)."""
    counts = np.zeros(3, np.int64)
    stl = 1 if ".stl" in str(path).lower() else 0
    null = (None,) * 6
    _check(lib().oracle_mesh_file_arrays(str(path).encode(), n, stl, ptr(counts, _L), *null))
    v, m, f = (int(x) for x in counts)
    out = {"vertices": np.zeros((v, n), np.float32), "normals": np.zeros((m, n), np.float32),
           "facet_vertices": np.zeros((f, n), np.int32), "facet_normals": np.zeros((f, n), np.int32),
           "has_normal": np.zeros(f, np.uint8), "facet_material": np.zeros(f, np.int32)}
    _check(lib().oracle_mesh_file_arrays(
        str(path).encode(), n, stl, ptr(counts, _L), ptr(out["vertices"], _F), ptr(out["normals"], _F),
        ptr(out["facet_vertices"], _I), ptr(out["facet_normals"], _I), ptr(out["has_normal"], _B),
        ptr(out["facet_material"], _I)))
    return out


# ---------------------------------------------------------------------------
# the reference's convex hull (oracle/_ref/libnbpt_hull.so, `make -C oracle
# hull`): 3-, 4- and 5-space (5-space with GMP integers)

HULL_PATH = HERE / "_ref" / "libnbpt_hull.so"
_hull = None


def hull_available() -> bool:
    return HULL_PATH.exists()


def convex_hull(points: np.ndarray) -> np.ndarray:
    """Facets [F][n] (vertex indices) of the reference's
    compute_convex_hull (src/geometry/core/convex_hull.h:95-98) of float
    points [count][n], n = 3, 4 or 5."""
    global _hull
    if _hull is None:
        if not HULL_PATH.exists():
            raise FileNotFoundError(f"hull library not built: {HULL_PATH} (run make -C oracle hull)")
        L = ctypes.CDLL(str(HULL_PATH))
        L.oracle_convex_hull.restype = ctypes.c_longlong
        L.oracle_convex_hull.argtypes = [ctypes.c_int, _F, ctypes.c_longlong, _I, ctypes.c_longlong]
        L.oracle_hull_error.restype = ctypes.c_char_p
        _hull = L
    p = np.ascontiguousarray(points, dtype=np.float32)
    count, n = p.shape
    cap = 16 * count + 64
    out = np.zeros((cap, n), np.int32)
    f = _hull.oracle_convex_hull(n, ptr(p, _F), count, ptr(out, _I), cap)
    if f < 0:
        raise OracleError(_hull.oracle_hull_error().decode())
    if f > cap:
        out = np.zeros((f, n), np.int32)
        f = _hull.oracle_convex_hull(n, ptr(p, _F), count, ptr(out, _I), f)
    return out[:f]
