"""Passes on the painter's worker thread with per-pass images through a
callback (the reference painter's thread and Notifier): the images equal
those of passes run one by one, passes are numbered from 1, stop ends the
worker early, and the painter refuses other calls while the worker runs."""

import threading
import time

import numpy as np
import pytest

from math_b200 import scenes

pytestmark = pytest.mark.gpu


def scene(painter):
    return painter.Scene(scenes.cornell_3d(size=(24, 24), subdivisions=3), "float", False)


def test_streamed_images_equal_sequential_passes(painter):
    s = scene(painter)
    ref = s.painter(16, 5, seed=9)
    expected = []
    for _ in range(4):
        ref.run(1)
        expected.append(ref.images())
    p = s.painter(16, 5, seed=9)
    got = []
    errors = []
    p.start(4, lambda k, rgb, rgba: got.append((k, rgb, rgba)), errors.append)
    p.join()
    assert not errors
    assert [k for k, _, _ in got] == [1, 2, 3, 4]
    for (_, rgb, rgba), (erg, erga) in zip(got, expected):
        assert np.array_equal(rgb, erg)
        assert np.array_equal(rgba, erga)
    assert not p.is_running()
    assert p.statistics()["pass_number"] == 4
    p.run(1)  # usable again once the worker ended


def test_stop_ends_an_unbounded_stream(painter):
    s = scene(painter)
    p = s.painter(16, 5, seed=2)
    seen = threading.Event()
    count = []

    def on_pass(k, rgb, rgba):
        count.append(k)
        seen.set()

    p.start(0, on_pass)
    assert seen.wait(60)
    assert p.is_running()
    with pytest.raises(painter.PainterError, match="worker thread"):
        p.run(1)
    p.stop()
    assert not p.is_running()
    n = len(count)
    time.sleep(0.2)
    assert len(count) == n >= 1
    assert count == list(range(1, n + 1))


def test_stream_errors(painter):
    s = scene(painter)
    p = s.painter(4, 5, seed=2)
    with pytest.raises(painter.PainterError, match="negative"):
        p.start(-1, lambda *a: None)
    L = painter.lib()
    assert L.nbpt_painter_start(p.h, 1, None, None, None) < 0
    assert "callback" in L.nbpt_last_error().decode()
