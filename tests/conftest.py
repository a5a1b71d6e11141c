"""Shared test configuration.

`-m "not gpu"` runs on any machine: the CPU restatement against the
reference's known-answer vectors, the oracle against the committed golden
fixtures, and the C ABI library's exports.  `-m gpu` runs the parity tests
of the CUDA path against the golden fixtures and, when it is built, the live
oracle (oracle/_ref/libnbpt_oracle.so).
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libnbpt.so")


@pytest.fixture(scope="session")
def golden():
    def load(name: str):
        with np.load(GOLDEN / f"{name}.npz") as f:
            return {k: f[k] for k in f.files}

    return load


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle

    if not oracle.available():
        pytest.skip("oracle library not built (make -C oracle)")
    return oracle


@pytest.fixture(scope="session")
def painter():
    from math_b200 import painter as p

    if p.device_count() < 1:
        pytest.fail("no CUDA device visible to the painter library")
    return p
