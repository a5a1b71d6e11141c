"""The C ABI library: it loads, exports every function include/nbpt.h
declares, and reports errors through status codes without a GPU."""

import ctypes
import re

import numpy as np
import pytest

from math_b200 import painter

from conftest import ROOT


def declared_functions() -> list[str]:
    text = (ROOT / "include" / "nbpt.h").read_text()
    return sorted(set(re.findall(r"\b(nbpt_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_the_binding_signatures():
    names = declared_functions()
    bound = sorted(name for name, _, _ in painter.SIGNATURES)
    assert names == bound


@pytest.mark.parametrize("c_name, mirror", [("nbpt_painter_options", painter.PainterOptions),
                                             ("nbpt_statistics", painter.Statistics),
                                             ("nbpt_job_info", painter.JobInfo)])
def test_header_structs_match_the_binding(c_name, mirror):
    """Every field of the header's struct, in order, in the ctypes mirror."""
    text = (ROOT / "include" / "nbpt.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    body = re.search(r"typedef struct %s\s*\{(.*?)\}\s*%s;" % (c_name, c_name), text, re.S)
    assert body, c_name
    fields = [re.findall(r"(\w+)\s*(?:\[\d+\])?\s*;", line)[0]
              for line in body.group(1).split("\n") if ";" in line]
    assert fields == [f[0] for f in mirror._fields_]


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(painter.LIB_PATH))
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_argument_errors_are_status_codes():
    L = painter.lib()
    assert L.nbpt_scene_create(7, 0, 0) is None
    assert b"dimension" in L.nbpt_last_error()
    assert L.nbpt_scene_create(3, 5, 0) is None
    h = L.nbpt_scene_create(3, 1, 0)
    assert h
    try:
        # a light on a shape that does not exist
        d = np.zeros(3)
        f = np.ones(3, np.float32)
        r = L.nbpt_scene_add_parallelotope_light(h, 4, d.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                 f.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
        assert r < 0
        assert b"hyperplane parallelotope" in L.nbpt_last_error()
        # finalizing without a projector
        assert L.nbpt_scene_finalize(h) < 0
    finally:
        L.nbpt_scene_destroy(h)


def test_painter_requires_a_finalized_scene():
    L = painter.lib()
    h = L.nbpt_scene_create(4, 0, 1)
    try:
        assert L.nbpt_painter_create(h, 16, 5, 1) is None
    finally:
        L.nbpt_scene_destroy(h)


def test_server_needs_a_device():
    L = painter.lib()
    if painter.device_count() > 0:
        pytest.skip("a GPU is present")
    assert L.nbpt_server_create(4, 0) is None
    assert b"device" in L.nbpt_last_error()
