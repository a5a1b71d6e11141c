"""Progress within a pass (nbpt_painter_set_progress), the counterpart of
the reference's per-pixel notifications (Notifier::pixel_set,
thread_busy / thread_free): after each chunk of a pass's pixels the callback
gets the pixels traced so far, in order, ending at the pass's pixel count;
and the chunk size (nbpt_painter_options.chunk_budget) changes no image."""

from __future__ import annotations

import numpy as np
import pytest

from math_b200 import painter as P
from math_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("integrator", ["bpt", "pt"])
def test_progress_per_chunk(painter, integrator):
    desc = scenes.cornell_4d(size=(12, 10, 9), points=500)
    s = P.Scene(desc, "float", False)
    whole = s.painter(16, 5, seed=3, integrator=integrator)
    whole.run(2)
    ref = whole.images()
    whole.close()
    # PT keeps no per-path buffers: its chunks bound the path counter only,
    # so it reports once per pass
    p = s.painter(16, 5, seed=3, integrator=integrator, chunk_budget=4 << 20)
    calls = []
    p.set_progress(lambda pass_, done, total: calls.append((pass_, done, total)))
    p.run(2)
    rgb, rgba = p.images()
    assert np.array_equal(rgb, ref[0]) and np.array_equal(rgba, ref[1])
    for k in (1, 2):
        mine = [c for c in calls if c[0] == k]
        assert mine, calls
        done = [c[1] for c in mine]
        assert all(b > a for a, b in zip(done, done[1:]))
        assert done[-1] == p.sources and all(c[2] == p.sources for c in mine)
        if integrator == "bpt":
            assert len(mine) > 2  # 4 MiB of chunk buffers: several chunks
    n = len(calls)
    p.set_progress(None)
    p.run(1)
    assert len(calls) == n
    p.close()
    s.close()


def test_negative_chunk_budget_is_rejected(painter):
    s = P.Scene(scenes.cornell_3d(size=(8, 8), subdivisions=1), "float", False)
    with pytest.raises(P.PainterError, match="negative"):
        s.painter(4, 3, chunk_budget=-1)
    s.close()
