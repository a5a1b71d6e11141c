"""The pixel estimator's group ordering (math_b200/csrc/group_order.h)
against libstdc++'s std::sort / std::partial_sort called as the reference's
src/painter/pixels/samples/com/sort.h calls them: the same permutation on
18,060 seeded groups of 0 to 300 entries, half of them full of equal keys
(tests/group_order_check.cpp, compiled here with g++)."""

import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_group_order_matches_libstdcxx(tmp_path):
    exe = tmp_path / "group_order_check"
    subprocess.run(["g++", "-std=c++20", "-O1", str(HERE / "group_order_check.cpp"), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    groups, mismatches = int(out[0]), int(out[1])
    assert groups == 18060
    assert mismatches == 0
