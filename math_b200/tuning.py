"""Measured choice of the job server's chunk budget.

A render's pass runs its paths in chunks of as many paths as its chunk
buffers hold (vertices, random-stream states, tapes and strategy queues:
about 6 KB per path at depth 8), and every chunk ends in a tail where the
persistent path kernels run out of paths and their blocks drain one lane at
a time.  With many renders on the GPU at once, each render's chunk budget is
a share of the server's memory budget: small shares mean short chunks and
long tails, large shares mean fewer renders at once to fill each other's
tails.  Which balance is best depends on the workload's mix of scene sizes,
so it is measured: `tune_chunk_budget` runs the caller's workload once per
candidate budget and keeps the fastest, and returns every trial for the log.
"""

from __future__ import annotations

import time
from typing import Callable

GIB = 1 << 30


def chunk_budget_candidates(server, factors=(1.0, 1.5, 2.0, 2.75), cap: int = 32 * GIB) -> list[int]:
    """Multiples of the server's default chunk budget (its memory budget's
    share per slot), at most `cap` (the painter's own upper bound)."""
    server.set_chunk_budget(0)
    base = server.chunk_budget
    out: list[int] = []
    for f in factors:
        b = min(cap, int(base * f))
        if b not in out:
            out.append(b)
    return out


def tune_chunk_budget(server, run: Callable[[], tuple[float, float]], candidates: list[int],
                      log: Callable[[str], None] | None = None, reset: Callable[[], object] | None = None) -> dict:
    """For each candidate (bytes): set it as the server's chunk budget, call
    `run()`, which renders a representative slice of the workload through the
    server and returns (paths, device seconds), and record paths/s.  The
    fastest candidate is left set.  `reset`, called before every trial and
    once more at the end, puts shared state back (the library's cache of
    device buffers, whose sizes follow the chunk budget: a cache filled by one
    candidate would slow the next, and the run after the tuning).  Returns
    {"chosen": bytes, "trials": [{"chunk_budget": bytes, "paths_per_s": r,
    "wall_s": w}, ...]}."""
    if not candidates:
        raise ValueError("no candidate chunk budgets")
    trials = []
    for b in candidates:
        if reset:
            reset()
        server.set_chunk_budget(b)
        t0 = time.perf_counter()
        paths, seconds = run()
        wall = time.perf_counter() - t0
        rate = paths / seconds if seconds > 0 else 0.0
        trials.append({"chunk_budget": int(b), "paths_per_s": rate, "wall_s": wall})
        if log:
            log(f"chunk budget {b / GIB:.2f} GiB: {rate / 1e6:.2f} M paths/s")
    best = max(trials, key=lambda t: t["paths_per_s"])
    server.set_chunk_budget(best["chunk_budget"])
    if reset:
        reset()
    return {"chosen": best["chunk_budget"], "trials": trials}
