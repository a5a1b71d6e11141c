"""Benchmark: bidirectional path tracing paths/s on one B200.

Workload (the configuration the headline metric is quoted on): the 4-space
Cornell box with a 3-sphere hull mesh (20,000 points on S^3, ~135k
3-simplex facets), a rotated 4-parallelotope and one 3-parallelotope light,
64-bin spectral colour, a 64x64x64 voxel screen, 16 requested samples per
voxel (27 rendered: the stratified sampler rounds up to 3^3), maximum path
depth 6.  Inputs are synthetic, generated from fixed seeds
(math_b200/scenes.py).

One step is one painter pass: every voxel's 27 paths traced, connected and
folded into the pixel estimator (7,077,888 paths).  `value` is paths/s over
the timed steps on the device (CUDA events on the painter's stream, L2
flushed between steps), `e2e` the same through the C ABI with the image read
back to host memory every step.  `--impl reference` runs the reference's own
CPU painter (compiled from its sources, oracle/_ref) on this machine's host
cores on a bounded slab of the same workload.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

# The single-scene workloads (the headline one first): scene, screen,
# samples per pixel, maximum depth, colour and the default precision.
WORKLOADS = {
    "cornell4d": {"screen": [64, 64, 64], "spp": 16, "max_depth": 6, "spectrum": True, "precision": "float",
                  "label": "4-space Cornell box, hull of 20000 points on S^3, spectrum64"},
    "cornell3d": {"screen": [256, 256], "spp": 16, "max_depth": 5, "spectrum": False, "precision": "double",
                  "label": "3-space Cornell box, icosphere of 20480 triangles, RGB"},
    "sphere4d": {"screen": [96, 96, 96], "spp": 8, "max_depth": 8, "spectrum": False, "precision": "float",
                 "label": "4-space hull of 150000 noisy points on S^3 (about 1M facets), ball light, "
                          "parallel projection, RGB"},
}


def workload_of(args) -> dict:
    return WORKLOADS[args.workload if args.workload in WORKLOADS else "cornell4d"]


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="nbpt", choices=["nbpt", "reference"])
    p.add_argument("--precision", default=None, choices=["float", "double"],
                   help="default: the workload's (float; double for cornell3d)")
    p.add_argument("--small", action="store_true", help="a small configuration for smoke runs")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--screen", type=int, default=None,
                   help="edge of the voxel screen (default: the workload's 64), for smaller profiling runs")
    p.add_argument("--workload", default="cornell4d", choices=["cornell4d", "cornell3d", "sphere4d", "batch", "serve", "meshfile"],
                   help="cornell4d: the headline benchmark; cornell3d, sphere4d: the other single-scene "
                        "workloads; batch: the mixed-scene batch, FP32 through the "
                        "job server against plain FP64 one job at a time; serve: Poisson arrivals of renders "
                        "into the job server, with completion latencies")
    p.add_argument("--integrator", default="bpt", choices=["bpt", "pt"],
                   help="single-scene workloads: bidirectional (the headline) or path tracing")
    p.add_argument("--jobs", type=int, default=64, help="batch: scenes in the batch")
    p.add_argument("--points-scale", type=float, default=1.0, help="batch/serve: scale of the hull point counts")
    p.add_argument("--screen-scale", type=float, default=1.0, help="batch/serve: scale of the screen edges")
    p.add_argument("--rate", type=float, default=40.0, help="serve: arrivals per second")
    p.add_argument("--duration", type=float, default=20.0, help="serve: seconds of arrivals")
    p.add_argument("--pool", type=int, default=16, help="serve: distinct scenes the jobs draw from")
    p.add_argument("--max-jobs", type=int, default=16, help="batch/serve: jobs the server runs at once")
    args = p.parse_args()
    if args.precision is None:
        args.precision = workload_of(args)["precision"]
    return args


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def scene_desc(small: bool, screen: int | None = None, name: str = "cornell4d"):
    from math_b200 import scenes

    w = WORKLOADS[name]
    dims = len(w["screen"])
    if small:
        size = tuple(max(4, e // 4) for e in w["screen"])
    else:
        size = tuple(w["screen"]) if screen is None else (screen,) * dims
    if name == "cornell4d":
        return scenes.cornell_4d(size=size, points=2000 if small else 20000)
    if name == "cornell3d":
        return scenes.cornell_3d(size=size, subdivisions=3 if small else 5)
    return scenes.sphere_4d(size=size, points=15000 if small else 150000)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return

        def read():
            for line in self.proc.stdout:
                self.rows.append([x.strip() for x in line.split(",")])

        self.thread = threading.Thread(target=read, daemon=True)
        self.thread.start()

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) < 9:
                continue
            for name, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(small: bool, name: str = "cornell4d", precision: str = "float", integrator: str = "bpt") -> dict:
    """The reference's own painter (create_painter with the integrator),
    unmodified, on the host cores: one pass over the workload's screen."""
    from math_b200 import scenes
    from oracle import oracle

    if not oracle.available():
        return {"value": None, "unit": "paths/s", "cores": 0, "kind": "reference",
                "sample": "oracle library not built"}
    # the whole workload: one pass over the full screen
    w = WORKLOADS[name]
    desc = scene_desc(small, None, name)
    slab = desc["projector"]["size"]
    s = oracle.Scene(desc, precision, w["spectrum"])
    s.set_integrator(integrator)
    cores = os.cpu_count() or 1
    stats, _ = s.paint(w["spp"], w["max_depth"], passes=1, threads=cores)
    value = stats["sample_count"] / stats["pass_duration"]
    return {"value": value, "unit": "paths/s", "cores": cores, "kind": "reference",
            "sample": (f"one pass of the reference painter over the whole {'x'.join(map(str, slab))} screen "
                       f"({stats['sample_count']} paths, {stats['pass_duration']:.2f} s, "
                       f"ray_count {stats['ray_count']})")}


# DRAM bytes (read + write) per path of the path kernels (walk, connect,
# light, replay) on this workload in float, from the ncu capture summarised
# in profiles/path_kernels_cornell4d_32.md (a 32^3 screen of the same scene;
# traffic scales with the number of paths)
TRAFFIC_PER_PATH = {"float": 20636.0}


def record_bytes(n: int, precision: str) -> dict:
    t = 8 if precision == "double" else 4
    return {"node": 2 * n * t + 8, "facet": n * (n + 1) * t + 4, "shape": n * (n + 1) * t}


def run_reference(args, rank: int):
    if rank != 0:
        return
    from math_b200 import scenes
    from oracle import oracle

    if not oracle.available():
        print(json.dumps({"impl": "reference", "unavailable": "the reference painter (oracle/_ref) is not built"}))
        return
    # --steps timed passes of the bounded slab (warm-up passes untimed)

    w = workload_of(args)
    desc = scene_desc(args.small, args.screen, args.workload if args.workload in WORKLOADS else "cornell4d")
    slab = desc["projector"]["size"]
    s = oracle.Scene(desc, args.precision, w["spectrum"])
    s.set_integrator(args.integrator)
    cores = os.cpu_count() or 1
    for _ in range(args.warmup):
        s.paint(w["spp"], w["max_depth"], passes=1, threads=cores)
    samples = 0
    seconds = 0.0
    for _ in range(args.steps):
        st, _ = s.paint(w["spp"], w["max_depth"], passes=1, threads=cores)
        samples += st["sample_count"]
        seconds += st["pass_duration"]
    value = samples / seconds
    sample = f"{args.steps} passes over the whole {'x'.join(map(str, slab))} screen"
    print(json.dumps({
        "metric": f"{args.integrator}_paths_per_second", "value": value, "unit": "paths/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * seconds / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "double" else "f32",
        "data": "synthetic (seeded generators)",
        "config": {"workload": f"{args.workload} {w['label']}, {w['spp']} spp, depth {w['max_depth']}",
                   "screen": slab, "precision": args.precision, "integrator": args.integrator},
        "cpu_baseline": {"value": value, "unit": "paths/s", "cores": cores, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "paths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def slowest_rank(seconds: float, world: int, device: str) -> float:
    """The largest of every rank's time (all ranks must call it)."""
    if world <= 1:
        return seconds
    import torch

    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank: float, world: int, seconds: float) -> float:
    """Whole-job throughput: every rank processed `units_per_rank` (weak
    scaling), timed by the slowest rank."""
    return world * units_per_rank / seconds


def run_nbpt(args, rank: int, world: int, local: int):
    import torch

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from math_b200 import painter as P

    w = workload_of(args)
    desc = scene_desc(args.small, args.screen, args.workload)
    spectrum = w["spectrum"]
    t0 = time.perf_counter()
    scene = P.Scene(desc, args.precision, spectrum)
    build_s = time.perf_counter() - t0
    # every rank renders its own pass sequence of the whole screen
    # (independent samples: weak scaling, no data-path collective)
    painter = scene.painter(w["spp"], w["max_depth"], seed=1 + rank, integrator=args.integrator)
    stream = torch.cuda.ExternalStream(painter_stream(painter))
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    for _ in range(args.warmup):
        painter.run(1)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()

    clocks = ClockSampler(local)
    clocks.start()
    # device-timed steps: events on the painter's stream around each pass,
    # L2 flushed between passes (outside the events)
    step_ms = []
    paths_s = 0.0
    nodes = facets = shapes = rays = launches = 0
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        painter.enqueue(1)
        end.record(stream)
        painter.wait()
        step_ms.append(start.elapsed_time(end))
        st = painter.statistics()
        paths_s += st["paths_seconds"]
        nodes += st["nodes"]
        facets += st["facets"]
        shapes += st["shapes"]
        rays += st["ray_count"]
        launches += st["kernel_launches"]
    torch.cuda.synchronize()
    clock_info = clocks.stop()

    paths_per_step = scene.pixels * painter.spp
    ms = slowest_rank(float(np.sum(step_ms)), world, "cuda")
    value = job_throughput(paths_per_step * args.steps, world, ms / 1000)

    # end to end through the C ABI, every step a whole job: the scene built
    # from host arrays (host->device copies, BVH build, facet setup on the
    # device), one pass, and the image read back to host memory
    rgb = np.zeros((scene.pixels, 3), np.float32)
    rgba = np.zeros((scene.pixels, 4), np.float32)
    torch.cuda.synchronize()
    e2e_times = []
    h2d = 0
    build = {}
    for _ in range(args.steps):
        e0 = time.perf_counter()
        job_scene = P.Scene(desc, args.precision, spectrum)
        job = job_scene.painter(w["spp"], w["max_depth"], seed=1 + rank, integrator=args.integrator)
        job.run(1)
        P._check(P.lib().nbpt_painter_images(job.h, P._p(rgb, P._F), P._p(rgba, P._F)))
        e2e_times.append(time.perf_counter() - e0)
        h2d = job_scene.upload_bytes()
        build = job_scene.build_seconds()
        job.close()
        job_scene.close()
    e2e_s = slowest_rank(float(np.sum(e2e_times)), world, "cuda")
    e2e = job_throughput(paths_per_step * args.steps, world, e2e_s)

    # scene resident: one pass through the C ABI plus the image read back
    torch.cuda.synchronize()
    r0 = time.perf_counter()
    for _ in range(args.steps):
        painter.run(1)
        P._check(P.lib().nbpt_painter_images(painter.h, P._p(rgb, P._F), P._p(rgba, P._F)))
    resident_s = time.perf_counter() - r0

    # scene resident, passes on the painter's worker thread, every pass's
    # images delivered to a callback while the next pass renders
    delivered = []
    noop = P.PASS_CALLBACK(lambda user, k, rgb, rgba, pixels: delivered.append(k))
    # one untimed pass pins the painter's host image buffers
    P._check(P.lib().nbpt_painter_start(painter.h, 1, P.ctypes.cast(noop, P.ctypes.c_void_p), None, None))
    P._check(P.lib().nbpt_painter_join(painter.h))
    delivered.clear()
    torch.cuda.synchronize()
    s0 = time.perf_counter()
    P._check(P.lib().nbpt_painter_start(painter.h, args.steps, P.ctypes.cast(noop, P.ctypes.c_void_p), None, None))
    P._check(P.lib().nbpt_painter_join(painter.h))
    streamed_s = time.perf_counter() - s0

    sizes = record_bytes(desc["n"], args.precision)
    algorithmic = nodes * sizes["node"] + facets * sizes["facet"] + shapes * sizes["shape"]
    achieved = algorithmic / paths_s / 1e9 if paths_s > 0 else None
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except (OSError, ValueError):
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None,
                "traffic": (TRAFFIC_PER_PATH[args.precision] * paths_per_step
                            if args.precision in TRAFFIC_PER_PATH and args.workload == "cornell4d"
                            and args.integrator == "bpt" and not args.small and args.screen is None else None),
                "traffic_source": "profiles/path_kernels_cornell4d_32.md (per path, scaled to one pass)",
                "kernel": ("path kernels (walk, connect, light, replay)" if args.integrator == "bpt"
                           else "pt_paths_kernel"),
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                "algorithmic_bytes_per_path": algorithmic / (paths_per_step * args.steps),
                "node_visits_per_path": nodes / (paths_per_step * args.steps),
                "facet_tests_per_path": facets / (paths_per_step * args.steps),
                "rays_per_path": rays / (paths_per_step * args.steps),
                "paths_kernel_share": paths_s / (ms / 1000) if ms > 0 else None}

    if rank == 0:
        cpu = (None if (args.no_cpu_baseline or world > 1)
               else cpu_baseline(args.small, args.workload, args.precision, args.integrator))
        line = {
            "metric": f"{args.integrator}_paths_per_second", "value": value, "unit": "paths/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "float" else "f64",
            "data": "synthetic (seeded generators)",
            "config": {"workload": f"{args.workload} {w['label']} ({scene.pixels} pixels), {w['spp']} spp "
                                   f"({painter.spp} rendered), depth {w['max_depth']}",
                       "screen": desc["projector"]["size"],
                       "paths_per_step": paths_per_step, "precision": args.precision,
                       "integrator": args.integrator,
                       "l2": "flushed (256 MiB write) between timed steps",
                       "scene_build_s": build_s},
            "e2e": {"value": e2e, "unit": "paths/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(rgb.nbytes + rgba.nbytes),
                    "seconds_per_step": e2e_s / args.steps,
                    "scene_build_seconds": build,
                    "note": "every step a whole job through the C ABI: scene from host arrays (copies, BVH "
                            "build, facet setup), one pass, RGB and RGBA images read back to host memory"},
            "resident": {"value": paths_per_step * args.steps / resident_s, "unit": "paths/s",
                         "note": "scene resident; one pass through the C ABI plus the image read back"},
            "streamed": {"value": paths_per_step * len(delivered) / streamed_s, "unit": "paths/s",
                         "note": "scene resident; passes on the painter's worker thread (nbpt_painter_start), "
                                 "each pass's RGB and RGBA images copied to pinned host memory and handed to a "
                                 "callback while the next pass renders"},
            "gpu_launches": launches,
            "roofline": roofline,
            "clocks": clock_info,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def painter_stream(painter) -> int:
    from math_b200 import painter as P

    return P.painter_stream(painter)


def rel_rmse(a, b) -> float:
    den = float((b.astype(np.float64) ** 2).sum())
    return float(np.sqrt(((a.astype(np.float64) - b) ** 2).sum() / den)) if den > 0 else 0.0


def run_batch(args):
    """The mixed-scene batch: every job rendered once (one pass of its
    samples per pixel) in FP64 one job at a time, then in FP32 through the
    job server, all jobs submitted at once; wall time of each whole batch
    with the scenes resident."""
    from math_b200 import painter as P
    from math_b200 import scenes

    t0 = time.perf_counter()
    jobs = scenes.mixed_batch(args.jobs, seed=4, points_scale=args.points_scale, screen_scale=args.screen_scale)
    generate_s = time.perf_counter() - t0
    fp64 = [P.Scene(j["desc"], "double", False) for j in jobs]
    fp32 = [P.Scene(j["desc"], "float", False) for j in jobs]
    paths = sum(s.pixels * s.actual_spp(j["spp"]) for s, j in zip(fp32, jobs))

    def plain():
        images = []
        for s, j in zip(fp64, jobs):
            p = s.painter(j["spp"], j["max_depth"], seed=1)
            p.run(1)
            images.append(p.images()[0])
            p.close()
        return images

    server = P.Server(max_jobs=args.max_jobs)
    try:
        batch_timed(args, server, jobs, fp64, fp32, paths, generate_s, plain)
    finally:
        server.close()


def batch_timed(args, server, jobs, fp64, fp32, paths, generate_s, plain):
    from math_b200 import scenes

    def batched():
        ids = [server.submit_render(s, j["spp"], j["max_depth"], seed=1, passes=1) for s, j in zip(fp32, jobs)]
        images = []
        for s, i in zip(fp32, ids):
            server.wait(i)
            images.append(server.images(i, s.pixels)[0])
            server.release(i)
        return images

    for _ in range(max(1, args.warmup)):
        batched()
    plain()
    t0 = time.perf_counter()
    ref = plain()
    plain_s = time.perf_counter() - t0
    best = None
    for _ in range(max(1, args.steps)):
        t0 = time.perf_counter()
        img = batched()
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    rmse = [rel_rmse(a, b) for a, b in zip(img, ref)]
    dims = [j["desc"]["n"] for j in jobs]
    line = {
        "metric": "batched_fp32_paths_per_second", "value": paths / best, "unit": "paths/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "plain_fp64": {"value": paths / plain_s, "seconds": plain_s,
                       "note": "one job at a time: painter, one pass, image read back"},
        "batched_fp32": {"value": paths / best, "seconds": best,
                         "note": f"all jobs submitted to the job server ({args.max_jobs} at once), "
                                 "created at admission, images read back; best of the timed batches"},
        "speedup_vs_plain_fp64": plain_s / best,
        "same_seed_rel_rmse_fp32_vs_fp64": {
            "median": float(np.median(rmse)), "max": float(np.max(rmse)),
            "note": "one pass each: float rounding moves paths off their double twins, so this is sample "
                    "noise, not bias; bias is tested against converged double images in tests/"},
        "dtype": "f32 (batched) / f64 (plain)", "data": "synthetic (seeded generators)",
        "config": {"workload": "mixed-scene batch: box, ceiling light and sphere hull in 3/4/5-space, RGB",
                   "jobs": len(jobs), "dims": {str(n): dims.count(n) for n in (3, 4, 5)},
                   "paths": paths, "facets_max": max(scenes.describe(j["desc"])["facets"] for j in jobs),
                   "points_scale": args.points_scale, "screen_scale": args.screen_scale,
                   "generate_s": generate_s},
    }
    print(json.dumps(line), flush=True)


def run_serve(args):
    """Poisson arrivals of renders into the job server: each job draws a
    scene from a pool of mixed-batch scenes (resident, FP32) and a sample
    budget log-uniform in [16, 256] samples per pixel; the server creates the
    render when it admits the job.  Latency is completion minus arrival."""
    from math_b200 import painter as P
    from math_b200 import scenes

    def note(msg):
        print(f"serve: {msg}", file=sys.stderr, flush=True)

    pool = scenes.mixed_batch(args.pool, seed=5, points_scale=args.points_scale, screen_scale=args.screen_scale)
    built = [P.Scene(j["desc"], "float", False) for j in pool]
    note(f"{len(built)} pool scenes built")
    rng = np.random.default_rng(5)
    arrivals = []
    t = 0.0
    while True:
        t += rng.exponential(1.0 / args.rate)
        if t > args.duration:
            break
        k = int(rng.integers(0, len(pool)))
        spp = int(round(math.exp(rng.uniform(math.log(16), math.log(256)))))
        # one pass renders at most 256 samples per pixel after the stratified
        # sampler rounds the count up to a power of the screen dimension
        while built[k].actual_spp(spp) > 256:
            spp -= 1
        arrivals.append((t, k, spp))
    server = P.Server(max_jobs=args.max_jobs)
    try:
        run_arrivals(args, server, pool, built, arrivals, note)
    finally:
        server.close()


def wait_with_watchdog(server, job, all_jobs, note, limit: float = 60.0):
    """Waits for a job by polling; if no job of the run progresses for
    `limit` seconds, reports every job's state and gives up."""
    last_change = time.perf_counter()
    last = None
    while True:
        info = server.job(job)
        if info["state"] in (2, 3):
            return server.wait(job)
        snapshot = [(j, server.job(j)["state"], server.job(j)["passes_done"]) for j in all_jobs]
        if snapshot != last:
            last = snapshot
            last_change = time.perf_counter()
        elif time.perf_counter() - last_change > limit:
            note("no progress: " + ", ".join(f"{j}:{st}/{pd}" for j, st, pd in snapshot))
            raise RuntimeError(f"job {job} made no progress for {limit} s")
        time.sleep(0.01)


def run_arrivals(args, server, pool, built, arrivals, note):
    """Submits the arrivals on their schedule, waits for every job and
    prints the serve line."""
    # warm-up: one render of every pool scene
    for s, j in zip(built, pool):
        i = server.submit_render(s, 4, j["max_depth"], seed=1)
        server.wait(i)
        server.release(i)
    note("warm-up done")
    t_start = server.time()
    submitted = []
    for a, k, spp in arrivals:
        while server.time() - t_start < a:
            time.sleep(min(0.001, max(0.0, a - (server.time() - t_start))))
        s = built[k]
        i = server.submit_render(s, spp, pool[k]["max_depth"], seed=len(submitted) + 1)
        submitted.append((i, t_start + a, s.pixels * s.actual_spp(spp)))
    note(f"{len(submitted)} jobs submitted")
    latencies, waits = [], []
    last = t_start
    pending = [j for j, _, _ in submitted]
    for i, arrival, _ in submitted:
        info = wait_with_watchdog(server, i, pending, note)
        pending.remove(i)
        latencies.append(info["finished"] - arrival)
        waits.append(info["started"] - arrival)
        last = max(last, info["finished"])
        server.release(i)
    paths = sum(p for _, _, p in submitted)
    lat = np.array(latencies)
    line = {
        "metric": "served_job_latency_p99", "value": float(np.percentile(lat, 99)), "unit": "s",
        "higher_is_better": False, "n_gpus": 1,
        "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
        "mean_queue_wait_s": float(np.mean(waits)),
        "jobs": len(submitted), "throughput_paths_per_second": paths / (last - t_start),
        "offered_paths_per_second": paths / args.duration,
        "makespan_s": last - t_start,
        "dtype": "f32", "data": "synthetic (seeded generators)",
        "config": {"workload": "Poisson render arrivals into the job server", "rate_per_s": args.rate,
                   "duration_s": args.duration, "pool_scenes": len(pool), "spp": "log-uniform 16-256",
                   "max_jobs": args.max_jobs, "points_scale": args.points_scale,
                   "screen_scale": args.screen_scale},
    }
    print(json.dumps(line), flush=True)


def run_meshfile(args):
    """Reading mesh files: a 4-space OBJ (with normals) and a binary STL of
    the convex hull of 50,000 points on S^3 (about 340,000 facets), parsed by
    nbpt_scene_add_mesh_file and by the reference's loaders (oracle), in
    file MB per second.  The library's figure includes turning the file's
    corners into the scene's points."""
    import tempfile

    sys.path.insert(0, str(ROOT / "tests"))
    from mesh_file_writers import write_obj, write_stl_binary
    from math_b200 import painter as P
    from math_b200 import scenes
    from oracle import oracle

    p, f = scenes.convex_hull_mesh(scenes.sphere_points(4, 50000 if not args.small else 2000, 8))
    p = np.asarray(p, np.float32)
    results = {}
    with tempfile.TemporaryDirectory() as d:
        files = {"obj4": Path(d) / "m.obj4", "stl4": Path(d) / "m.stl4"}
        write_obj(files["obj4"], p, f, normals=p / np.linalg.norm(p, axis=1, keepdims=True))
        write_stl_binary(files["stl4"], p, f)
        L = P.lib()
        m = np.eye(5).reshape(-1)
        rgb = np.array([0.5, 0.5, 0.5], np.float32)
        for name, path in files.items():
            size_mb = path.stat().st_size / 1e6
            ours = []
            ref = []
            for _ in range(args.warmup + args.steps):
                h = L.nbpt_scene_create(4, 0, 0)
                t0 = time.perf_counter()
                P._check(L.nbpt_scene_add_mesh_file(h, str(path).encode(), P._p(m, P._D), 0.0, 0.3,
                                                    P._p(rgb, P._F), 1.0))
                ours.append(time.perf_counter() - t0)
                L.nbpt_scene_destroy(h)
                if oracle.available():
                    t0 = time.perf_counter()
                    oracle.load_mesh_file(path, 4)
                    ref.append(time.perf_counter() - t0)
            ours = ours[args.warmup:]
            ref = ref[args.warmup:]
            results[name] = {"file_mb": size_mb, "facets": int(len(f)),
                             "nbpt_mb_per_s": size_mb / float(np.median(ours)),
                             "reference_mb_per_s": size_mb / float(np.median(ref)) if ref else None}
    first = results["obj4"]
    print(json.dumps({
        "metric": "mesh_file_mb_per_second", "value": first["nbpt_mb_per_s"], "unit": "MB/s",
        "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators)",
        "config": {"workload": "4-space OBJ with normals (value) and binary STL of a hull of 50,000 points on S^3",
                   "files": results},
        "cpu_baseline": {"value": first["reference_mb_per_s"], "unit": "MB/s", "cores": os.cpu_count(),
                         "kind": "reference", "sample": "the reference's load_from_obj_file on the same file"},
    }), flush=True)


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.workload == "batch":
        if rank == 0:
            run_batch(args)
        return
    if args.workload == "serve":
        if rank == 0:
            run_serve(args)
        return
    if args.workload == "meshfile":
        if rank == 0:
            run_meshfile(args)
        return
    run_nbpt(args, rank, world, local)


if __name__ == "__main__":
    main()
