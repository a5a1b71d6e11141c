"""The job server (nbpt_server_*): renders that run together through it give
the same images, bit for bit, as each render alone, since every path's
random stream depends only on (seed, pass, pixel, sample)."""

from __future__ import annotations

import numpy as np
import pytest

from math_b200 import painter as P
from math_b200 import scenes


@pytest.mark.gpu
def test_server_results_match_renders_alone(painter):
    jobs = scenes.mixed_batch(6, seed=7, points_scale=0.02, screen_scale=0.1)
    passes = 2
    alone = []
    for j in jobs:
        s = P.Scene(j["desc"], "float", False)
        p = s.painter(j["spp"], j["max_depth"], seed=3)
        p.run(passes)
        alone.append(p.images())
        p.close()
        s.close()

    server = P.Server(max_jobs=4)
    held = []
    ids = []
    for j in jobs:
        s = P.Scene(j["desc"], "float", False)
        p = s.painter(j["spp"], j["max_depth"], seed=3)
        held.append((s, p))
        ids.append(server.submit(p, passes))
    for k, (job_id, (s, p)) in enumerate(zip(ids, held)):
        info = server.wait(job_id)
        assert info["state"] == 2  # NBPT_JOB_DONE
        assert info["passes_done"] == passes
        assert 0 <= info["submitted"] <= info["started"] <= info["finished"]
        assert info["footprint"] > 0
        rgb, rgba = p.images()
        assert np.array_equal(rgb, alone[k][0])
        assert np.array_equal(rgba, alone[k][1])
        assert p.statistics()["pass_number"] == passes
    server.close()
    for s, p in held:
        p.close()
        s.close()


@pytest.mark.gpu
def test_server_admits_jobs_within_its_slots(painter):
    jobs = scenes.mixed_batch(5, seed=9, points_scale=0.01, screen_scale=0.08)
    server = P.Server(max_jobs=2)
    held = [(s := P.Scene(j["desc"], "float", False), s.painter(j["spp"], j["max_depth"], seed=1)) for j in jobs]
    ids = [server.submit(p, 3) for _, p in held]
    infos = [server.wait(i) for i in ids]
    # never more than two jobs between admission and completion at once
    events = sorted([(i["started"], 1) for i in infos] + [(i["finished"], -1) for i in infos],
                    key=lambda e: (e[0], e[1]))
    running = 0
    for _, d in events:
        running += d
        assert running <= 2
    with pytest.raises(P.PainterError):
        server.submit(held[0][1], 0)
    server.close()
    for s, p in held:
        p.close()
        s.close()


@pytest.mark.gpu
def test_server_created_renders_match_renders_alone(painter):
    jobs = scenes.mixed_batch(4, seed=11, points_scale=0.02, screen_scale=0.1)
    built = [P.Scene(j["desc"], "float", False) for j in jobs]
    alone = []
    for s, j in zip(built, jobs):
        p = s.painter(j["spp"], j["max_depth"], seed=5)
        p.run(1)
        alone.append(p.images()[0])
        p.close()
    server = P.Server(max_jobs=3)
    ids = [server.submit_render(s, j["spp"], j["max_depth"], seed=5, passes=1) for s, j in zip(built, jobs)]
    for k, job_id in enumerate(ids):
        info = server.wait(job_id)
        assert info["state"] == 2
        rgb, _ = server.images(job_id, built[k].pixels)
        assert np.array_equal(rgb, alone[k])
        assert server.statistics(job_id)["sample_count"] == built[k].pixels * built[k].actual_spp(jobs[k]["spp"])
        server.release(job_id)
    with pytest.raises(P.PainterError):
        server.job(ids[0])  # released
    server.close()
    for s in built:
        s.close()


@pytest.mark.gpu
def test_chunk_budget_changes_no_image(painter):
    """Renders the server creates with a small chunk budget (many chunks per
    pass) equal those with the default, bit for bit: every path's stream,
    tape and strategies are its own, so chunk boundaries change nothing."""
    jobs = scenes.mixed_batch(3, seed=11, points_scale=0.02, screen_scale=0.1)
    built = [P.Scene(j["desc"], "float", False) for j in jobs]
    server = P.Server(max_jobs=3)
    default = server.chunk_budget
    assert default >= 4 << 30
    images = {}
    launches = {}
    for budget in (0, 8 << 20):
        server.set_chunk_budget(budget)
        assert server.chunk_budget == (budget or default)
        ids = [server.submit_render(s, j["spp"], j["max_depth"], seed=5, passes=2) for s, j in zip(built, jobs)]
        out = []
        for s, i in zip(built, ids):
            assert server.wait(i)["state"] == 2
            out.append(server.images(i, s.pixels))
            launches.setdefault(budget, []).append(server.statistics(i)["kernel_launches"])
            server.release(i)
        images[budget] = out
    # 8 MiB of chunk buffers hold fewer paths than a pass of the larger jobs
    assert any(b > a for a, b in zip(launches[0], launches[8 << 20]))
    for a, b in zip(images[0], images[8 << 20]):
        assert np.array_equal(a[0], b[0])
        assert np.array_equal(a[1], b[1])
    with pytest.raises(P.PainterError, match="negative"):
        server.set_chunk_budget(-1)
    server.close()
    for s in built:
        s.close()
