"""Python binding of the painter's C ABI (include/nbpt.h, math_b200/libnbpt.so).

    scene = Scene(description, precision="double", spectrum=False)
    painter = scene.painter(samples_per_pixel=16, max_depth=5, seed=1)
    painter.run(passes=1)
    rgb, rgba = painter.images()

A scene description is the dict format of math_b200.scenes.  Every render
runs on the GPU: the library has no CPU path, and loading it without its
built shared object raises.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libnbpt.so"

_lib = None

_P = ctypes.c_void_p
_D = ctypes.POINTER(ctypes.c_double)
_F = ctypes.POINTER(ctypes.c_float)
_I = ctypes.POINTER(ctypes.c_int)
_U = ctypes.POINTER(ctypes.c_uint)
_B = ctypes.POINTER(ctypes.c_ubyte)
_L = ctypes.POINTER(ctypes.c_longlong)


class JobInfo(ctypes.Structure):
    _fields_ = [
        ("state", ctypes.c_int),
        ("passes", ctypes.c_int),
        ("passes_done", ctypes.c_int),
        ("footprint", ctypes.c_longlong),
        ("submitted", ctypes.c_double),
        ("started", ctypes.c_double),
        ("finished", ctypes.c_double),
        ("device_started", ctypes.c_double),
        ("device_finished", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class PainterOptions(ctypes.Structure):
    _fields_ = [
        ("integrator", ctypes.c_int),
        ("samples_per_pixel", ctypes.c_int),
        ("max_depth", ctypes.c_int),
        ("seed", ctypes.c_uint),
        ("flat_shading", ctypes.c_int),
        ("slab_begin", ctypes.c_int),
        ("slab_end", ctypes.c_int),
        ("pixel_sums", ctypes.c_int),
        ("chunk_budget", ctypes.c_longlong),
    ]


class Statistics(ctypes.Structure):
    _fields_ = [
        ("pass_number", ctypes.c_longlong),
        ("pixel_count", ctypes.c_longlong),
        ("ray_count", ctypes.c_longlong),
        ("sample_count", ctypes.c_longlong),
        ("previous_pass_duration", ctypes.c_double),
        ("paths_seconds", ctypes.c_double),
        ("nodes", ctypes.c_ulonglong),
        ("facets", ctypes.c_ulonglong),
        ("shapes", ctypes.c_ulonglong),
        ("kernel_launches", ctypes.c_longlong),
        ("nonfinite_samples", ctypes.c_longlong),
        ("stack_overflows", ctypes.c_longlong),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


# (name, restype, argtypes) of every exported function, in include/nbpt.h order
SIGNATURES = [
    ("nbpt_last_error", ctypes.c_char_p, []),
    ("nbpt_release_cached_memory", ctypes.c_longlong, []),
    ("nbpt_device_count", ctypes.c_int, []),
    ("nbpt_scene_create", _P, [ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("nbpt_scene_destroy", None, [_P]),
    ("nbpt_scene_add_hyperplane_parallelotope", ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, _F, ctypes.c_double, _D, _D]),
    ("nbpt_scene_add_parallelotope", ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, _F, ctypes.c_double, _D, _D]),
    ("nbpt_scene_add_mesh_object", ctypes.c_int, [_P, _F, ctypes.c_longlong, _I, ctypes.c_longlong, _D, _F, ctypes.c_float, ctypes.c_float, _F, ctypes.c_float]),
    ("nbpt_scene_add_mesh", ctypes.c_int, [_P]),
    ("nbpt_scene_add_mesh_data", ctypes.c_int, [_P, ctypes.c_longlong, _D, _D, ctypes.c_longlong, _I, _I, ctypes.c_int, _D, _F]),
    ("nbpt_scene_add_parallelotope_light", ctypes.c_int, [_P, ctypes.c_int, _D, _F]),
    ("nbpt_scene_add_ball_light", ctypes.c_int, [_P, _D, _D, ctypes.c_double, _F]),
    ("nbpt_scene_set_perspective_projector", ctypes.c_int, [_P, _D, _D, _D, ctypes.c_double, _I]),
    ("nbpt_scene_set_parallel_projector", ctypes.c_int, [_P, _D, _D, _D, ctypes.c_double, _I]),
    ("nbpt_scene_set_background", ctypes.c_int, [_P, _F]),
    ("nbpt_scene_finalize", ctypes.c_int, [_P]),
    ("nbpt_scene_pixel_count", ctypes.c_longlong, [_P]),
    ("nbpt_scene_actual_spp", ctypes.c_int, [_P, ctypes.c_int]),
    ("nbpt_scene_device_bytes", ctypes.c_longlong, [_P]),
    ("nbpt_scene_upload_bytes", ctypes.c_longlong, [_P]),
    ("nbpt_scene_build_seconds", ctypes.c_int, [_P, _D]),
    ("nbpt_scene_add_mesh_file", ctypes.c_int,
     [_P, ctypes.c_char_p, _D, ctypes.c_float, ctypes.c_float, _F, ctypes.c_float]),
    ("nbpt_mesh_file_dimension", ctypes.c_int, [ctypes.c_char_p]),
    ("nbpt_scene_set_bvh_builder", ctypes.c_int, [_P, ctypes.c_int]),
    ("nbpt_painter_create", _P, [_P, ctypes.c_int, ctypes.c_int, ctypes.c_uint]),
    ("nbpt_painter_create_integrator", _P, [_P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint]),
    ("nbpt_painter_create_slab", _P, [_P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint, ctypes.c_int, ctypes.c_int]),
    ("nbpt_painter_create_options", _P, [_P, ctypes.POINTER(PainterOptions)]),
    ("nbpt_painter_destroy", None, [_P]),
    ("nbpt_painter_start", ctypes.c_int, [_P, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, _P]),
    ("nbpt_painter_stop", ctypes.c_int, [_P]),
    ("nbpt_painter_join", ctypes.c_int, [_P]),
    ("nbpt_painter_is_running", ctypes.c_int, [_P]),
    ("nbpt_painter_enqueue", ctypes.c_int, [_P, ctypes.c_int]),
    ("nbpt_painter_wait", ctypes.c_int, [_P]),
    ("nbpt_painter_images", ctypes.c_int, [_P, _F, _F]),
    ("nbpt_painter_samples", ctypes.c_int, [_P, _D, _F, _B]),
    ("nbpt_painter_statistics", ctypes.c_int, [_P, ctypes.POINTER(Statistics)]),
    ("nbpt_painter_stream", _P, [_P]),
    ("nbpt_painter_cancel", ctypes.c_int, [_P]),
    ("nbpt_painter_set_progress", ctypes.c_int, [_P, ctypes.c_void_p, _P]),
    ("nbpt_server_create", _P, [ctypes.c_int, ctypes.c_longlong]),
    ("nbpt_server_destroy", None, [_P]),
    ("nbpt_server_submit", ctypes.c_longlong, [_P, _P, ctypes.c_int]),
    ("nbpt_server_submit_render", ctypes.c_longlong, [_P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_uint, ctypes.c_int]),
    ("nbpt_server_images", ctypes.c_int, [_P, ctypes.c_longlong, _F, _F]),
    ("nbpt_server_statistics", ctypes.c_int, [_P, ctypes.c_longlong, ctypes.POINTER(Statistics)]),
    ("nbpt_server_release", ctypes.c_int, [_P, ctypes.c_longlong]),
    ("nbpt_server_job", ctypes.c_int, [_P, ctypes.c_longlong, ctypes.POINTER(JobInfo)]),
    ("nbpt_server_wait", ctypes.c_int, [_P, ctypes.c_longlong, ctypes.POINTER(JobInfo)]),
    ("nbpt_server_time", ctypes.c_double, [_P]),
    ("nbpt_server_cancel", ctypes.c_int, [_P, ctypes.c_longlong]),
    ("nbpt_server_set_chunk_budget", ctypes.c_int, [_P, ctypes.c_longlong]),
    ("nbpt_server_chunk_budget", ctypes.c_longlong, [_P]),
    ("nbpt_scene_trace", ctypes.c_int, [_P, _D, ctypes.c_longlong, ctypes.c_int, _I, _I, _D, _D]),
    ("nbpt_scene_trace_noalloc", ctypes.c_int, [_P, _D, ctypes.c_longlong, ctypes.c_int, _I, _I, _D, _D]),
    ("nbpt_scene_mesh_export", ctypes.c_int, [_P, ctypes.c_int, _L, _D, _D, _D, _U, _U, _I]),
    ("nbpt_scene_ingested_mesh", ctypes.c_int, [_P, ctypes.c_int, _L, _D, _D, _I]),
    ("nbpt_scene_brdf", ctypes.c_int, [_P, ctypes.c_int, _D, _D, _D, _F, _D]),
    ("nbpt_scene_brdf_sample", ctypes.c_int, [_P, ctypes.c_int, _D, _D, _U, ctypes.c_int, _D, _D, _F]),
    ("nbpt_scene_light_sample", ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, _U, ctypes.c_int, _D, _D, _F]),
    ("nbpt_test_server_fail_allocations", ctypes.c_int, [_P, ctypes.c_int]),
    ("nbpt_test_server_hold", ctypes.c_int, [_P, ctypes.c_int]),
    ("nbpt_test_pcg", ctypes.c_int, [_U, ctypes.c_int, ctypes.c_int, _U]),
    ("nbpt_test_canonical", ctypes.c_int, [_U, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D]),
    ("nbpt_test_sj_points", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _U, ctypes.c_int, _D]),
    ("nbpt_test_bvh_build", ctypes.c_int, [ctypes.c_int, ctypes.c_int, _D, ctypes.c_longlong, _I, ctypes.c_longlong, _L, _I]),
]


class PainterError(RuntimeError):
    pass


def lib():
    """The loaded C ABI library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise PainterError(f"{LIB_PATH} is not built: run __graft_entry__.build() or make -C math_b200/csrc")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(r):
    if r is None or (isinstance(r, int) and r < 0):
        raise PainterError(lib().nbpt_last_error().decode())
    return r


def _d(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _f(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _i(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def _null(t):
    return ctypes.cast(None, t)


def _seed(words):
    w = np.ascontiguousarray(np.asarray(words, dtype=np.uint32))
    return w, len(w)


class Scene:
    """A scene on the GPU built from a scene description (math_b200.scenes).

    mesh_data: optional list, one entry per mesh shape in order, of the
    painter's mesh data (vertices, normals, facets, facet_material,
    material_params, material_colors) used instead of the shape's mesh
    objects; lets a caller render exactly the mesh another painter prepared.
    """

    def __init__(self, desc: dict, precision: str = "float", spectrum: bool = False,
                 mesh_data: list | None = None, bvh_builder: str = "device"):
        L = lib()
        self.n = int(desc["n"])
        self.spectrum = bool(spectrum)
        self.channels = 64 if spectrum else 3
        self.precision = precision
        self.h = L.nbpt_scene_create(self.n, 1 if precision == "double" else 0, 1 if spectrum else 0)
        if not self.h:
            raise PainterError(L.nbpt_last_error().decode())
        n = self.n
        mesh_index = 0
        for s in desc["shapes"]:
            kind = s["type"]
            if kind == "hyperplane_parallelotope":
                _check(L.nbpt_scene_add_hyperplane_parallelotope(
                    self.h, s["metalness"], s["roughness"], _p(_f(s["color"]), _F), s["alpha"],
                    _p(_d(s["org"]), _D), _p(_d(s["vectors"]).reshape(-1), _D)))
            elif kind == "parallelotope":
                _check(L.nbpt_scene_add_parallelotope(
                    self.h, s["metalness"], s["roughness"], _p(_f(s["color"]), _F), s["alpha"],
                    _p(_d(s["org"]), _D), _p(_d(s["vectors"]).reshape(-1), _D)))
            elif kind == "mesh":
                if mesh_data is not None:
                    m = mesh_data[mesh_index]
                    v = _d(m["vertices"]).reshape(-1, n)
                    nm = m.get("normals")
                    nm = _d(nm).reshape(-1, n) if nm is not None and len(nm) else None
                    fc = _i(m["facets"]).reshape(-1, n)
                    fm = _i(m["facet_material"])
                    mp = _d(m["material_params"]).reshape(-1, 3)
                    mc = _f(m["material_colors"]).reshape(len(mp), -1)
                    _check(L.nbpt_scene_add_mesh_data(
                        self.h, len(v), _p(v, _D), _p(nm, _D) if nm is not None else _null(_D), len(fc),
                        _p(fc, _I), _p(fm, _I), len(mp), _p(mp, _D), _p(mc, _F)))
                else:
                    for o in s["objects"]:
                        if "file" in o:
                            _check(L.nbpt_scene_add_mesh_file(
                                self.h, str(o["file"]).encode(), _p(_d(o["matrix"]).reshape(-1), _D),
                                o["metalness"], o["roughness"], _p(_f(o["color"]), _F), o["alpha"]))
                            continue
                        pts = _f(o["points"]).reshape(-1, n)
                        fac = _i(o["facets"]).reshape(-1, n)
                        nrm = o.get("normals")
                        nrm = _f(nrm).reshape(-1, n) if nrm is not None else None
                        _check(L.nbpt_scene_add_mesh_object(
                            self.h, _p(pts, _F), len(pts), _p(fac, _I), len(fac),
                            _p(_d(o["matrix"]).reshape(-1), _D),
                            _p(nrm, _F) if nrm is not None else _null(_F),
                            o["metalness"], o["roughness"], _p(_f(o["color"]), _F), o["alpha"]))
                    _check(L.nbpt_scene_add_mesh(self.h))
                mesh_index += 1
            else:
                raise ValueError(f"unknown shape type {kind}")
        for l in desc["lights"]:
            if l["type"] == "parallelotope":
                _check(L.nbpt_scene_add_parallelotope_light(
                    self.h, l["shape"], _p(_d(l["direction"]), _D), _p(_f(l["radiance"]), _F)))
            elif l["type"] == "ball":
                _check(L.nbpt_scene_add_ball_light(
                    self.h, _p(_d(l["center"]), _D), _p(_d(l["direction"]), _D), l["radius"],
                    _p(_f(l["radiance"]), _F)))
            else:
                raise ValueError(f"unknown light type {l['type']}")
        p = desc["projector"]
        size = _i(p["size"])
        if p["type"] == "perspective":
            _check(L.nbpt_scene_set_perspective_projector(
                self.h, _p(_d(p["org"]), _D), _p(_d(p["dir"]), _D),
                _p(_d(p["axes"]).reshape(-1), _D), p["fov"], _p(size, _I)))
        else:
            _check(L.nbpt_scene_set_parallel_projector(
                self.h, _p(_d(p["org"]), _D), _p(_d(p["dir"]), _D),
                _p(_d(p["axes"]).reshape(-1), _D), p["units_per_pixel"], _p(size, _I)))
        _check(L.nbpt_scene_set_background(self.h, _p(_f(desc["background"]), _F)))
        _check(L.nbpt_scene_set_bvh_builder(self.h, {"device": 0, "host": 1}[bvh_builder]))
        _check(L.nbpt_scene_finalize(self.h))
        self.size = [int(x) for x in p["size"]]
        self.pixels = int(np.prod(self.size))

    def close(self):
        h = getattr(self, "h", None)
        if h and _lib is not None:
            _lib.nbpt_scene_destroy(h)
        self.h = None

    def __del__(self):
        self.close()

    def actual_spp(self, spp: int) -> int:
        return _check(lib().nbpt_scene_actual_spp(self.h, spp))

    def device_bytes(self) -> int:
        return _check(lib().nbpt_scene_device_bytes(self.h))

    def upload_bytes(self) -> int:
        return _check(lib().nbpt_scene_upload_bytes(self.h))

    def build_seconds(self) -> dict:
        """Host seconds of the build: mesh ingestion, BVH builds, the rest of
        finalize (device uploads, facet setup) and the total."""
        out = np.zeros(4)
        _check(lib().nbpt_scene_build_seconds(self.h, _p(out, _D)))
        return dict(zip(("ingest", "bvh", "upload", "total"), (float(x) for x in out)))

    def painter(self, samples_per_pixel: int, max_depth: int, seed: int = 1,
                integrator: str = "bpt", slab: tuple[int, int] | None = None,
                flat_shading: bool = False, pixel_sums: str | None = None, chunk_budget: int = 0) -> "Painter":
        """slab: rows [begin, end) of the last screen axis (nbpt_painter_create_slab);
        flat_shading: create_painter's flat_shading; pixel_sums: "float",
        "double" or None (float for a double-precision scene, else double);
        chunk_budget: bytes of per-chunk path buffers (0: the default)"""
        return Painter(self, samples_per_pixel, max_depth, seed, integrator, slab, flat_shading, pixel_sums,
                       chunk_budget)

    def trace(self, rays: np.ndarray, any_hit: bool = False):
        rays = _d(rays).reshape(-1, 2 * self.n)
        m = len(rays)
        kind = np.zeros(m, np.int32)
        index = np.zeros(m, np.int32)
        t = np.zeros(m)
        point = np.zeros((m, self.n))
        _check(lib().nbpt_scene_trace(self.h, _p(rays, _D), m, 1 if any_hit else 0, _p(kind, _I),
                                      _p(index, _I), _p(t, _D), _p(point, _D)))
        if any_hit:
            return kind.astype(bool)
        return kind, index, t, point

    def mesh_export(self, mesh: int = 0) -> dict:
        n = self.n
        counts = np.zeros(3, np.int64)
        L = lib()
        _check(L.nbpt_scene_mesh_export(self.h, mesh, _p(counts, _L), _null(_D), _null(_D), _null(_D),
                                        _null(_U), _null(_U), _null(_I)))
        nf, nodes, ni = (int(c) for c in counts)
        out = {"planes": np.zeros((nf, n, n + 1)), "node_lo": np.zeros((nodes, n)),
               "node_hi": np.zeros((nodes, n)), "node_info": np.zeros((nodes, 3), np.uint32),
               "indices": np.zeros(ni, np.uint32), "normal_info": np.zeros((nf, 2), np.int32)}
        _check(L.nbpt_scene_mesh_export(self.h, mesh, _p(counts, _L), _p(out["planes"], _D),
                                        _p(out["node_lo"], _D), _p(out["node_hi"], _D),
                                        _p(out["node_info"], _U), _p(out["indices"], _U),
                                        _p(out["normal_info"], _I)))
        return out

    def brdf(self, material: int, n, v, l):
        f = np.zeros(self.channels, np.float32)
        pdf = np.zeros(1)
        _check(lib().nbpt_scene_brdf(self.h, material, _p(_d(n), _D), _p(_d(v), _D), _p(_d(l), _D),
                                     _p(f, _F), _p(pdf, _D)))
        return f, float(pdf[0])

    def brdf_sample(self, material: int, n, v, seed_words):
        w, k = _seed(seed_words)
        l = np.zeros(self.n)
        pdf = np.zeros(1)
        f = np.zeros(self.channels, np.float32)
        _check(lib().nbpt_scene_brdf_sample(self.h, material, _p(_d(n), _D), _p(_d(v), _D), _p(w, _U), k,
                                            _p(l, _D), _p(pdf, _D), _p(f, _F)))
        return l, float(pdf[0]), f

    def light_sample(self, light: int, kind: str, seed_words, point=None):
        w, k = _seed(seed_words)
        out = np.zeros(3 * self.n + 2)
        rad = np.zeros(self.channels, np.float32)
        point = _d(point if point is not None else np.zeros(self.n))
        _check(lib().nbpt_scene_light_sample(self.h, light, 0 if kind == "leave" else 1, _p(w, _U), k,
                                             _p(point, _D), _p(out, _D), _p(rad, _F)))
        return out, rad


# painter::Integrator (src/painter/painter.h:143-147)
INTEGRATORS = {"bpt": 0, "pt": 1}
# NBPT_PIXEL_SUMS_*: the type of the estimator's per-pixel sums; None is the
# default (float for a double-precision scene, double for a single-precision one)
PIXEL_SUMS = {None: 0, "float": 1, "double": 2}

PASS_CALLBACK = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_longlong, ctypes.POINTER(ctypes.c_float),
                                 ctypes.POINTER(ctypes.c_float), ctypes.c_longlong)
ERROR_CALLBACK = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_char_p)
PROGRESS_CALLBACK = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_longlong)


class Painter:
    """One render of a scene (the reference's create_painter): integrator
    "bpt" (bidirectional, max_depth bounds the subpaths) or "pt" (path
    tracing with next-event estimation; max_depth is not used)."""

    def __init__(self, scene: Scene, samples_per_pixel: int, max_depth: int, seed: int = 1,
                 integrator: str = "bpt", slab: tuple[int, int] | None = None, flat_shading: bool = False,
                 pixel_sums: str | None = None, chunk_budget: int = 0):
        if integrator not in INTEGRATORS:
            raise PainterError(f"Unknown integrator {integrator!r}")
        if pixel_sums not in PIXEL_SUMS:
            raise PainterError(f"Unknown pixel sums {pixel_sums!r}")
        self.scene = scene
        self.integrator = integrator
        self.spp = scene.actual_spp(samples_per_pixel)
        begin, end = slab if slab is not None else (0, -1)
        options = PainterOptions(INTEGRATORS[integrator], samples_per_pixel, max_depth, seed,
                                 1 if flat_shading else 0, begin, end, PIXEL_SUMS[pixel_sums], int(chunk_budget))
        self.h = lib().nbpt_painter_create_options(scene.h, ctypes.byref(options))
        if not self.h:
            raise PainterError(lib().nbpt_last_error().decode())
        # receiving pixels (the slab) and the pixels whose paths a pass renders
        rows = scene.size[-1]
        row = scene.pixels // rows
        if slab is None:
            self.pixels = self.sources = scene.pixels
        else:
            self.pixels = (end - begin) * row
            self.sources = (min(rows, end + 1) - max(0, begin - 1)) * row

    def close(self):
        h = getattr(self, "h", None)
        if h and _lib is not None:
            _lib.nbpt_painter_destroy(h)
        self.h = None
        self._callbacks = None

    def start(self, max_passes: int, on_pass, on_error=None):
        """Runs `max_passes` passes (0: until stop()) on the painter's worker
        thread; on_pass(pass, rgb [P, 3], rgba [P, 4]) gets each pass's images
        (copies) while the next pass renders; on_error(message) a failure."""

        def pass_cb(user, pass_number, rgb, rgba, pixels):
            a = np.ctypeslib.as_array(rgb, shape=(pixels, 3)).copy()
            b = np.ctypeslib.as_array(rgba, shape=(pixels, 4)).copy()
            on_pass(int(pass_number), a, b)

        def error_cb(user, message):
            if on_error is not None:
                on_error(message.decode())

        c_pass = PASS_CALLBACK(pass_cb)
        c_error = ERROR_CALLBACK(error_cb)
        self._callbacks = (c_pass, c_error)  # kept alive while the worker runs
        _check(lib().nbpt_painter_start(self.h, max_passes, ctypes.cast(c_pass, ctypes.c_void_p),
                                        ctypes.cast(c_error, ctypes.c_void_p), None))

    def stop(self):
        _check(lib().nbpt_painter_stop(self.h))

    def join(self):
        _check(lib().nbpt_painter_join(self.h))

    def is_running(self) -> bool:
        return _check(lib().nbpt_painter_is_running(self.h)) == 1

    def cancel(self):
        _check(lib().nbpt_painter_cancel(self.h))

    def set_progress(self, fn):
        """fn(pass, pixels_done, pixels) after each chunk of a pass's paths
        (nbpt_painter_set_progress; it runs on a CUDA host-callback thread);
        None removes it."""
        if fn is None:
            _check(lib().nbpt_painter_set_progress(self.h, None, None))
            self._progress = None
            return
        cb = PROGRESS_CALLBACK(lambda user, p, done, total: fn(int(p), int(done), int(total)))
        _check(lib().nbpt_painter_set_progress(self.h, ctypes.cast(cb, ctypes.c_void_p), None))
        self._progress = cb

    def __del__(self):
        self.close()

    def enqueue(self, passes: int = 1):
        _check(lib().nbpt_painter_enqueue(self.h, passes))

    def wait(self):
        _check(lib().nbpt_painter_wait(self.h))

    def run(self, passes: int = 1):
        self.enqueue(passes)
        self.wait()

    def images(self):
        rgb = np.zeros((self.pixels, 3), np.float32)
        rgba = np.zeros((self.pixels, 4), np.float32)
        _check(lib().nbpt_painter_images(self.h, _p(rgb, _F), _p(rgba, _F)))
        return rgb, rgba

    def samples(self):
        P, S, n = self.sources, self.spp, self.scene.n
        points = np.zeros((P, S, n - 1))
        colors = np.zeros((P, S, self.scene.channels), np.float32)
        valid = np.zeros((P, S), np.uint8)
        _check(lib().nbpt_painter_samples(self.h, _p(points, _D), _p(colors, _F), _p(valid, _B)))
        return points, colors, valid.astype(bool)

    def statistics(self) -> dict:
        s = Statistics()
        _check(lib().nbpt_painter_statistics(self.h, ctypes.byref(s)))
        return s.as_dict()


def painter_stream(p: "Painter") -> int:
    """The painter's CUDA stream handle (cudaStream_t as an integer)."""
    return int(lib().nbpt_painter_stream(p.h) or 0)


def release_cached_memory() -> int:
    """Frees the device buffers the library keeps for reuse (nbpt_release_cached_memory); returns their bytes."""
    return _check(lib().nbpt_release_cached_memory())


def device_count() -> int:
    return lib().nbpt_device_count()


def test_pcg(seed_words, count: int) -> np.ndarray:
    w, k = _seed(seed_words)
    out = np.zeros(count, np.uint32)
    _check(lib().nbpt_test_pcg(_p(w, _U), k, count, _p(out, _U)))
    return out


def test_canonical(seed_words, count: int, double: bool = True) -> np.ndarray:
    w, k = _seed(seed_words)
    out = np.zeros(count)
    _check(lib().nbpt_test_canonical(_p(w, _U), k, count, 1 if double else 0, _p(out, _D)))
    return out


def test_sj_points(dimension: int, spp: int, seed_words, double: bool = True) -> np.ndarray:
    w, k = _seed(seed_words)
    count = _check(lib().nbpt_test_sj_points(dimension, 1 if double else 0, spp, _p(w, _U), k, _null(_D)))
    out = np.zeros((count, dimension))
    _check(lib().nbpt_test_sj_points(dimension, 1 if double else 0, spp, _p(w, _U), k, _p(out, _D)))
    return out


class Server:
    """Continuous batching of renders on one GPU (nbpt_server_*): every
    admitted job keeps one pass in flight on its painter's stream; jobs
    submitted while others run are admitted as slots and memory free up."""

    def __init__(self, max_jobs: int = 16, memory_budget: int = 0):
        self.h = lib().nbpt_server_create(max_jobs, memory_budget)
        if not self.h:
            raise PainterError(lib().nbpt_last_error().decode())

    def submit(self, painter: "Painter", passes: int = 1) -> int:
        return _check(lib().nbpt_server_submit(self.h, painter.h, passes))

    def submit_render(self, scene: "Scene", samples_per_pixel: int, max_depth: int, seed: int = 1,
                      passes: int = 1) -> int:
        return _check(lib().nbpt_server_submit_render(self.h, scene.h, samples_per_pixel, max_depth, seed, passes))

    def images(self, job: int, pixels: int):
        rgb = np.zeros((pixels, 3), np.float32)
        rgba = np.zeros((pixels, 4), np.float32)
        _check(lib().nbpt_server_images(self.h, job, _p(rgb, _F), _p(rgba, _F)))
        return rgb, rgba

    def statistics(self, job: int) -> dict:
        st = Statistics()
        _check(lib().nbpt_server_statistics(self.h, job, ctypes.byref(st)))
        return st.as_dict()

    def release(self, job: int):
        _check(lib().nbpt_server_release(self.h, job))

    def job(self, job: int) -> dict:
        info = JobInfo()
        _check(lib().nbpt_server_job(self.h, job, ctypes.byref(info)))
        return info.as_dict()

    def wait(self, job: int) -> dict:
        info = JobInfo()
        _check(lib().nbpt_server_wait(self.h, job, ctypes.byref(info)))
        return info.as_dict()

    def time(self) -> float:
        return lib().nbpt_server_time(self.h)

    def cancel(self, job: int):
        _check(lib().nbpt_server_cancel(self.h, job))

    def set_chunk_budget(self, nbytes: int):
        """Chunk-buffer bytes of the renders submitted from now on (0: the default share per slot)."""
        _check(lib().nbpt_server_set_chunk_budget(self.h, int(nbytes)))

    @property
    def chunk_budget(self) -> int:
        return _check(lib().nbpt_server_chunk_budget(self.h))

    def try_wait(self, job: int) -> dict:
        """wait() that returns the failed job's info (with "error") instead of raising."""
        info = JobInfo()
        r = lib().nbpt_server_wait(self.h, job, ctypes.byref(info))
        d = info.as_dict()
        d["error"] = lib().nbpt_last_error().decode() if r < 0 else None
        return d

    def hold_admission(self, hold: bool):
        """test hook: while held the server admits no job"""
        _check(lib().nbpt_test_server_hold(self.h, 1 if hold else 0))

    def fail_next_allocations(self, count: int):
        """test hook: the next `count` renders created at admission fail as out of device memory"""
        _check(lib().nbpt_test_server_fail_allocations(self.h, count))

    def close(self):
        h = getattr(self, "h", None)
        if h and _lib is not None:
            _lib.nbpt_server_destroy(h)
        self.h = None

    def __del__(self):
        self.close()
