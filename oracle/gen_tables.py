"""Writes tables.inc: numeric tables the painter's arithmetic depends on.

The values must be identical to the reference's, so they are read out of the
reference itself, through the CPU oracle (oracle/_ref/libnbpt_oracle.so, built
from the reference sources by oracle/Makefile), and written as C++ arrays:

  * the n-D GGX single-scattering directional-albedo tables for n = 3, 4, 5:
    32x32 over (cosine, roughness) and 32 cosine-weighted averages over
    roughness, in float and in double (src/shading/ggx/f1_albedo.cpp);
  * the 64-bin spectral basis over 380-720 nm: CIE 1931 x, y, z colour
    matching functions and the seven reflectance and seven D65 illumination
    Smits basis spectra (src/color/color.h:156-210).

Run from the repository root when the oracle is built:
    python -m oracle.gen_tables
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from oracle import oracle  # noqa: E402


def fmt(values, kind: str) -> str:
    if kind == "float":
        items = [np.format_float_scientific(np.float32(v), unique=True) + "f" for v in values]
    else:
        items = [repr(float(v)) for v in values]
    lines = []
    for i in range(0, len(items), 6):
        lines.append("        " + ", ".join(items[i:i + 6]) + ",")
    return "\n".join(lines)


def main() -> None:
    out = []
    out.append("// Generated by oracle/gen_tables.py from the reference painter's own")
    out.append("// tables (read through the CPU oracle).  Do not edit by hand.")
    out.append("// clang-format off")
    out.append("#pragma once")
    out.append("")
    out.append("namespace nbpt::tables")
    out.append("{")
    for n in (3, 4, 5):
        tf, af, td, ad = oracle.f1_albedo_tables(n)
        out.append(f"// n = {n}: f1 albedo, [roughness][cosine] (cosine fastest), and its cosine-weighted average")
        out.append(f"inline constexpr float F1_ALBEDO_{n}_F[1024] = {{")
        out.append(fmt(tf, "float"))
        out.append("};")
        out.append(f"inline constexpr float F1_AVERAGE_{n}_F[32] = {{")
        out.append(fmt(af, "float"))
        out.append("};")
        out.append(f"inline constexpr double F1_ALBEDO_{n}_D[1024] = {{")
        out.append(fmt(td, "double"))
        out.append("};")
        out.append(f"inline constexpr double F1_AVERAGE_{n}_D[32] = {{")
        out.append(fmt(ad, "double"))
        out.append("};")
    s = oracle.spectrum_functions()
    names = ["CIE_X", "CIE_Y", "CIE_Z",
             "REFLECTANCE_WHITE", "REFLECTANCE_CYAN", "REFLECTANCE_MAGENTA", "REFLECTANCE_YELLOW",
             "REFLECTANCE_RED", "REFLECTANCE_GREEN", "REFLECTANCE_BLUE",
             "ILLUMINATION_WHITE", "ILLUMINATION_CYAN", "ILLUMINATION_MAGENTA", "ILLUMINATION_YELLOW",
             "ILLUMINATION_RED", "ILLUMINATION_GREEN", "ILLUMINATION_BLUE"]
    out.append("// 64 spectral bins over 380-720 nm")
    out.append("inline constexpr double SPECTRUM[17][64] = {")
    for name, row in zip(names, s):
        out.append(f"        {{ // {name}")
        out.append(fmt(row, "double"))
        out.append("        },")
    out.append("};")
    out.append("}")
    out.append("// clang-format on")
    (ROOT / "math_b200" / "csrc" / "tables.inc").write_text("\n".join(out) + "\n")


if __name__ == "__main__":
    main()
