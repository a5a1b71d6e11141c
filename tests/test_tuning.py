"""The chunk-budget tuner (math_b200/tuning.py) against a stand-in server:
candidates are multiples of the default capped at the painter's bound, each
candidate is measured once, and the fastest is left set."""

from __future__ import annotations

import pytest

from math_b200 import tuning as T


class FakeServer:
    def __init__(self, default: int):
        self.default = default
        self.budget = 0
        self.history = []

    def set_chunk_budget(self, b: int):
        self.budget = b
        self.history.append(b)

    @property
    def chunk_budget(self) -> int:
        return self.budget or self.default


def test_candidates_are_capped_multiples_of_the_default():
    s = FakeServer(9 * T.GIB)
    c = T.chunk_budget_candidates(s)
    assert c == [9 * T.GIB, int(13.5 * T.GIB), 18 * T.GIB, int(24.75 * T.GIB)]
    big = FakeServer(20 * T.GIB)
    assert T.chunk_budget_candidates(big) == [20 * T.GIB, 30 * T.GIB, 32 * T.GIB]


def test_the_fastest_candidate_is_kept():
    s = FakeServer(9 * T.GIB)
    rates = {9: 60.0, 16: 64.0, 24: 58.0}
    seen = []

    def run():
        gib = s.budget // T.GIB
        seen.append(gib)
        return rates[gib] * 10.0, 10.0

    resets = []
    out = T.tune_chunk_budget(s, run, [9 * T.GIB, 16 * T.GIB, 24 * T.GIB], log=lambda m: None,
                              reset=lambda: resets.append(s.budget))
    assert seen == [9, 16, 24]
    # before every trial (with the previous budget still set) and at the end
    assert len(resets) == 4 and resets[-1] == 16 * T.GIB
    assert out["chosen"] == 16 * T.GIB
    assert s.budget == 16 * T.GIB
    assert [t["paths_per_s"] for t in out["trials"]] == [60.0, 64.0, 58.0]
    with pytest.raises(ValueError):
        T.tune_chunk_budget(s, run, [])
