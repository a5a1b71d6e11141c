"""Failure paths, injected on the host (no device fault): cancelling a queued
or running job and a painter (the reference's stop flag,
src/painter/painting/integrator_bpt.cpp:90-93, and Painter's destructor,
painter.cpp:129-134), running out of device memory at admission (a failure
the server's test hook injects), scenes the build refuses, jobs whose render
cannot be created, and infinite radiance in the scene input, whose samples
are counted as the reference logs them (pixels.cpp:107-113); a NaN radiance
becomes 0 when the colour is built, max(0, NaN), in both.  Every failure
is reported through a status code and nbpt_last_error, and the server goes
on with its other jobs."""

from __future__ import annotations

import time

import numpy as np
import pytest

from math_b200 import painter as P
from math_b200 import scenes

pytestmark = pytest.mark.gpu


def small_scene(size=16, precision="float"):
    return P.Scene(scenes.cornell_3d(size=(size, size), subdivisions=2), precision, False)


def large_scene():
    # about 7 M paths per pass: a pass lasts long enough to be cancelled in flight
    return P.Scene(scenes.cornell_4d(size=(64, 64, 64), points=2000), "float", False)


def render_alone(scene, spp, depth, seed):
    p = scene.painter(spp, depth, seed=seed)
    p.run(1)
    rgb = p.images()[0]
    p.close()
    return rgb


def test_cancel_a_queued_job(painter):
    big = large_scene()
    small = small_scene()
    server = P.Server(max_jobs=1)
    a = server.submit_render(big, 16, 6, seed=1)
    b = server.submit_render(small, 16, 5, seed=2)
    server.cancel(b)
    info = server.try_wait(b)
    assert info["state"] == 3  # NBPT_JOB_FAILED
    assert "cancelled" in info["error"]
    assert info["started"] == -1
    done = server.try_wait(a)
    assert done["state"] == 2 and done["error"] is None
    server.release(a)
    server.release(b)
    server.close()


def test_cancel_a_running_job_and_go_on(painter):
    big = large_scene()
    small = small_scene()
    expected = render_alone(small, 16, 5, seed=4)
    server = P.Server(max_jobs=2)
    a = server.submit_render(big, 16, 6, seed=1, passes=50)
    while server.job(a)["state"] != 1:
        time.sleep(0.001)
    time.sleep(0.05)
    t0 = time.perf_counter()
    server.cancel(a)
    info = server.try_wait(a)
    waited = time.perf_counter() - t0
    assert info["state"] == 3
    assert "cancelled" in info["error"]
    assert info["passes_done"] < 50
    assert waited < 5.0
    # the server runs the next job as if nothing had happened
    b = server.submit_render(small, 16, 5, seed=4)
    assert server.try_wait(b)["state"] == 2
    rgb, _ = server.images(b, small.pixels)
    assert np.array_equal(rgb, expected)
    server.cancel(b)  # a finished job is left as it is
    assert server.job(b)["state"] == 2
    server.release(a)
    server.release(b)
    server.close()


def test_cancel_a_painter_mid_pass(painter):
    big = large_scene()
    p = big.painter(16, 6, seed=1)
    p.enqueue(20)
    p.cancel()
    with pytest.raises(P.PainterError, match="cancelled"):
        p.wait()
    with pytest.raises(P.PainterError, match="cancelled"):
        p.enqueue(1)
    p.close()


def test_cancel_a_painter_worker(painter):
    big = large_scene()
    p = big.painter(16, 6, seed=1)
    errors = []
    p.start(0, lambda k, rgb, rgba: None, errors.append)
    time.sleep(0.05)
    p.cancel()
    p.join()
    assert not p.is_running()
    assert any("cancelled" in e for e in errors)
    p.close()


def test_out_of_memory_at_admission_keeps_arrival_order(painter):
    jobs = scenes.mixed_batch(4, seed=13, points_scale=0.02, screen_scale=0.1)
    built = [P.Scene(j["desc"], "float", False) for j in jobs]
    alone = [render_alone(s, j["spp"], j["max_depth"], seed=6) for s, j in zip(built, jobs)]
    big = large_scene()
    server = P.Server(max_jobs=3)
    # a long job holds a slot, so a render that finds the device full is not
    # running alone (one that is fails at once: nothing would free memory)
    blocker = server.submit_render(big, 16, 6, seed=1, passes=1000)
    while server.job(blocker)["state"] != 1:
        time.sleep(0.001)
    # the four renders queue while admission is held; when it resumes the
    # first two are admitted together and both find the device full
    server.hold_admission(True)
    ids = [server.submit_render(s, j["spp"], j["max_depth"], seed=6) for s, j in zip(built, jobs)]
    server.fail_next_allocations(2)
    server.hold_admission(False)
    time.sleep(0.2)
    assert all(server.job(i)["state"] == 0 for i in ids)  # all queued again: nothing admitted since
    server.cancel(blocker)
    assert "cancelled" in server.try_wait(blocker)["error"]
    infos = [server.try_wait(i) for i in ids]
    # every render ran: the ones that found the device full went back to the
    # head of the queue, and admission kept the arrival order
    assert all(i["state"] == 2 for i in infos), infos
    started = [i["started"] for i in infos]
    assert started == sorted(started), [(i["submitted"], i["started"], i["finished"]) for i in infos]
    for k, i in enumerate(ids):
        rgb, _ = server.images(i, built[k].pixels)
        assert np.array_equal(rgb, alone[k])
        server.release(i)
    server.release(blocker)
    server.close()


def test_a_render_that_cannot_be_created_fails_alone(painter):
    s = small_scene()
    server = P.Server(max_jobs=2)
    bad = server.submit_render(s, 16, 9, seed=1)  # depth beyond 8
    good = server.submit_render(s, 16, 5, seed=1)
    info = server.try_wait(bad)
    assert info["state"] == 3
    assert "maximum depth" in info["error"]
    assert server.try_wait(good)["state"] == 2
    server.close()


def test_scene_the_build_refuses(painter):
    desc = scenes.cornell_3d(size=(8, 8), subdivisions=1)
    mesh = [s for s in desc["shapes"] if s["type"] == "mesh"][0]
    mesh["objects"][0]["facets"] = np.array(mesh["objects"][0]["facets"]).copy()
    mesh["objects"][0]["facets"][3, 1] = 10 ** 6
    with pytest.raises(P.PainterError, match="out of range"):
        P.Scene(desc, "float", False)
    no_light = scenes.cornell_3d(size=(8, 8), subdivisions=1)
    no_light["lights"] = []
    with pytest.raises(P.PainterError, match="No light sources"):
        P.Scene(no_light, "float", False)


@pytest.mark.parametrize("precision", ["float", "double"])
def test_non_finite_radiance_is_counted(painter, precision):
    desc = scenes.cornell_3d(size=(12, 12), subdivisions=2)
    desc["lights"][0]["radiance"] = [float("inf"), 1.0, 1.0]
    s = P.Scene(desc, precision, False)
    p = s.painter(16, 5, seed=1)
    p.run(1)
    st = p.statistics()
    assert st["nonfinite_samples"] > 0
    assert st["stack_overflows"] == 0
    p.run(1)  # counted over the painter's passes
    assert p.statistics()["nonfinite_samples"] > st["nonfinite_samples"]
    # a finite scene counts none
    q = small_scene(12, precision).painter(16, 5, seed=1)
    q.run(1)
    assert q.statistics()["nonfinite_samples"] == 0
