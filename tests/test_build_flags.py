"""The library's compile options: every unit but the single-precision path
kernels' (painter_paths_f.cu) is compiled without multiply-add contraction
on device and host, which double precision's bit-exactness rests on; only
that unit takes contraction, flushed denormals and approximate division and
square root.  Checked on the Makefile, without a GPU."""

from __future__ import annotations

import re

from conftest import ROOT

MAKEFILE = ROOT / "math_b200" / "csrc" / "Makefile"


def variable(text: str, name: str) -> str:
    m = re.search(r"^%s\s*:?=\s*((?:.*\\\n)*.*)$" % re.escape(name), text, re.M)
    assert m, name
    return m.group(1).replace("\\\n", " ")


def test_exact_units_compile_without_contraction():
    text = MAKEFILE.read_text()
    nvcc = variable(text, "NVCCFLAGS")
    assert "-fmad=false" in nvcc and "-ffp-contract=off" in nvcc
    for fast in ("-fmad=true", "-ftz=true", "-prec-div=false", "-prec-sqrt=false", "use_fast_math"):
        assert fast not in nvcc
    assert "-ffp-contract=off" in variable(text, "CXXFLAGS")


def test_only_the_single_precision_path_unit_is_fast():
    text = MAKEFILE.read_text()
    rules = re.findall(r"^(\$\(OBJ\)/[^:\n]+):[^\n]*\n\t[^\n]*\n\t([^\n]*)", text, re.M)
    fast = [target for target, recipe in rules if "-fmad=true" in recipe]
    assert fast == ["$(OBJ)/painter_paths_f.o"]
    recipe = dict(rules)["$(OBJ)/painter_paths_f.o"]
    for option in ("-fmad=true", "-ftz=true", "-prec-div=false", "-prec-sqrt=false"):
        assert option in recipe
    # and the unit holds only the single-precision path kernels
    unit = (ROOT / "math_b200" / "csrc" / "painter_paths_f.cu").read_text()
    assert "<N, double>" not in unit and "double" not in re.sub(r"//.*", "", unit)
