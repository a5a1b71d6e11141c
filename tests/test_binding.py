"""The reference-side binding (tests/binding/nbpt_painter.h: a
painter::Painter over the C ABI, as INTEGRATION.md shows it), compiled
against the reference's own painter.h by oracle/Makefile, driven by a
Notifier that records every call (tests/binding/binding_check.cpp): passes
numbered from 1 with their images, images equal to the C ABI painter's,
argument errors thrown, an unbounded painter stopped by its destructor."""

import subprocess

import pytest

from conftest import ROOT

BINARY = ROOT / "oracle" / "_ref" / "binding_check"


@pytest.mark.gpu
def test_reference_side_binding(painter):
    if not BINARY.exists():
        pytest.skip("binding test program not built (make -C oracle binding)")
    r = subprocess.run([str(BINARY)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "binding ok" in r.stdout


def test_binding_program_links_the_library():
    if not BINARY.exists():
        pytest.skip("binding test program not built (make -C oracle binding)")
    # without a GPU the program reaches the scene build and reports the device
    r = subprocess.run([str(BINARY)], capture_output=True, text=True, timeout=120)
    from math_b200 import painter as P

    if P.device_count() == 0:
        assert r.returncode == 1 and "no CUDA device" in r.stdout
