"""Benchmark: bidirectional path tracing paths/s on one B200.

Headline workload (the default, `--workload batch`): the mixed-scene batch
the metric is quoted on.  64 scenes (seed 4), dimension uniform in
{3, 4, 5}: a box of parallelotope walls, one parallelotope light and the
convex hull of N points on the unit (n-1)-sphere (N log-uniform in
[2k, 200k]; 5-space hulls capped at 50k points), screens 128^2-512^2,
32^3-96^3 or 16^4-32^4, 4-64 samples per pixel log-uniform, maximum depth
5-8, RGB.  Inputs are synthetic, generated from fixed seeds
(math_b200/scenes.py).

One step is one wave, a quarter of the batch's jobs (about 192 M of its
770 M paths), one pass each through the job server in FP32, all submitted
at once.  With `--tune` the server's chunk budget is chosen by measurement
before the warm-up (math_b200.tuning).  `value` is paths/s over the timed
steps on the device (CUDA events on the jobs' streams, each step's first
kernel to its last, L2 flushed between steps); `plain_fp64` the same jobs in
FP64 one at a time;
`e2e` the whole batch through the C ABI from host arrays (scene builds,
copies, images back); `serve` a Poisson stream of renders into the server
with its p50/p99 latency.  `--impl reference` runs the reference's own CPU
painter (compiled from its sources, oracle/_ref) on this machine's host
cores, one job at a time, on bounded samples of every job.

The single-scene workloads (`cornell4d`, `cornell3d`, `sphere4d`) time
painter passes of one scene the same way.
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
                 "label": "4-space hull of 150000 noisy points on S^3 (321,175 facets), ball light, "
                          "parallel projection, RGB"},
    "mixed5d": {"screen": [12, 12, 12, 12], "spp": 16, "max_depth": 8, "spectrum": False, "precision": "float",
                "label": "a 5-space job of the mixed batch's shape: box, ceiling light, hull of 24000 points on S^4 "
                         "(739,992 facets), RGB (for kernel profiles)"},
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
    p.add_argument("--workload", default="batch", choices=["batch", "cornell4d", "cornell3d", "sphere4d", "mixed5d", "serve", "meshfile"],
                   help="batch (the headline): the 64-scene mixed batch, FP32 through the job server against "
                        "plain FP64 one job at a time, with a served stream beside it; cornell4d, cornell3d, "
                        "sphere4d: single-scene workloads; serve: Poisson arrivals of renders into the job server "
                        "at --rate for --duration; meshfile: OBJ / STL reading")
    p.add_argument("--integrator", default="bpt", choices=["bpt", "pt"],
                   help="single-scene workloads: bidirectional (the headline) or path tracing")
    p.add_argument("--jobs", type=int, default=64, help="batch: scenes in the batch")
    p.add_argument("--points-scale", type=float, default=1.0, help="batch/serve: scale of the hull point counts")
    p.add_argument("--screen-scale", type=float, default=1.0, help="batch/serve: scale of the screen edges")
    p.add_argument("--rate", type=float, default=40.0, help="serve: arrivals per second")
    p.add_argument("--duration", type=float, default=20.0, help="serve: seconds of arrivals")
    p.add_argument("--pool", type=int, default=16, help="serve: distinct scenes the jobs draw from")
    p.add_argument("--max-jobs", type=int, default=16, help="batch/serve: jobs the server runs at once")
    p.add_argument("--waves", type=int, default=4,
                   help="batch: the batch is split into this many waves of about equal paths; a step is one wave")
    p.add_argument("--tune", action="store_true",
                   help="batch: choose the server's chunk budget by measurement (math_b200.tuning, one batch per "
                        "candidate, before the warm-up) instead of keeping its default; on this batch the "
                        "candidates differ by less than one batch's run-to-run spread")
    p.add_argument("--e2e-steps", type=int, default=0,
                   help="batch: steps (waves) of the end-to-end measurement (0: one whole batch)")
    p.add_argument("--serve-duration", type=float, default=20.0,
                   help="batch: seconds of arrivals of the served stream beside it (0: none)")
    p.add_argument("--serve-load", type=float, default=0.7,
                   help="batch: offered load of that stream, as a fraction of the measured batched throughput")
    p.add_argument("--ref-target", type=int, default=1000000,
                   help="batch: paths per job of the reference painter's bounded samples")
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
    if name == "mixed5d":
        return scenes.mixed_scene(5, 2400 if small else 24000, list(size), 4056)
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
    cores = os.cpu_count() or 1
    # in a watchdog child: the reference painter can stall at the end of a pass
    (paths, seconds), = reference_job_passes(desc, w["spp"], w["max_depth"], 1, cores, precision=precision,
                                             spectrum=w["spectrum"], integrator=integrator)[0]
    value = paths / seconds
    return {"value": value, "unit": "paths/s", "cores": cores, "kind": "reference",
            "sample": (f"one pass of the reference painter over the whole {'x'.join(map(str, slab))} screen "
                       f"({paths} paths, {seconds:.2f} s)")}


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
    cores = os.cpu_count() or 1
    # warm-up and timed passes in a watchdog child: the reference painter can
    # stall at the end of a pass (reference_job_passes)
    passes, _ = reference_job_passes(desc, w["spp"], w["max_depth"], args.warmup + args.steps, cores,
                                     precision=args.precision, spectrum=w["spectrum"],
                                     integrator=args.integrator)
    timed = passes[args.warmup:]
    samples = sum(p for p, _ in timed)
    seconds = sum(t for _, t in timed)
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
    # one render split across the ranks by slabs of the screen (math_b200/
    # tiles.py): each rank renders its slab's paths and its halo rows', no
    # collective while rendering, one gather of the slab images at the end
    from math_b200 import tiles

    rows = desc["projector"]["size"][-1]
    slab = tiles.slab_rows(rows, rank, world) if world > 1 else None
    painter = scene.painter(w["spp"], w["max_depth"], seed=1, integrator=args.integrator, slab=slab)
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

    # the screen's paths per step, all ranks together (the halo rows' second
    # rendering is not counted)
    paths_per_step = scene.pixels * painter.spp
    ms = slowest_rank(float(np.sum(step_ms)), world, "cuda")
    value = paths_per_step * args.steps / (ms / 1000)

    # end to end through the C ABI, every step a whole job: the scene built
    # from host arrays (host->device copies, BVH build, facet setup on the
    # device), one pass, and the image read back to host memory
    rgb = np.zeros((painter.pixels, 3), np.float32)
    rgba = np.zeros((painter.pixels, 4), np.float32)
    torch.cuda.synchronize()
    e2e_times = []
    h2d = 0
    build = {}
    for _ in range(args.steps):
        e0 = time.perf_counter()
        job_scene = P.Scene(desc, args.precision, spectrum)
        job = job_scene.painter(w["spp"], w["max_depth"], seed=1, integrator=args.integrator, slab=slab)
        job.run(1)
        P._check(P.lib().nbpt_painter_images(job.h, P._p(rgb, P._F), P._p(rgba, P._F)))
        if world > 1:
            # the slab images gathered into the whole image on rank 0
            tiles.gather_image(rgb, rank, world, rows, desc["projector"]["size"])
        e2e_times.append(time.perf_counter() - e0)
        h2d = job_scene.upload_bytes()
        build = job_scene.build_seconds()
        job.close()
        job_scene.close()
    e2e_s = slowest_rank(float(np.sum(e2e_times)), world, "cuda")
    e2e = paths_per_step * args.steps / e2e_s

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
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
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
            "resident": {"value": painter.pixels * painter.spp * args.steps / resident_s, "unit": "paths/s",
                         "note": "scene resident; one pass through the C ABI plus the image read back"},
            "streamed": {"value": painter.pixels * painter.spp * len(delivered) / streamed_s, "unit": "paths/s",
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


# ---------------------------------------------------------------------------
# The headline workload: 64 mixed scenes in 3/4/5-space (seed 4), batched
# FP32 through the job server against the plain FP64 path one job at a time

BATCH_SEED = 4
SERVE_SEED = 5
BATCH_LABEL = ("mixed-scene batch: 64 scenes, dimension uniform in {3,4,5}, box of parallelotope walls, one "
               "parallelotope light and the convex hull of N points on the unit (n-1)-sphere (N log-uniform in "
               "[2k, 200k], 5-space capped at 50k), screens 128^2-512^2 / 32^3-96^3 / 16^4-32^4, 4-64 spp "
               "log-uniform (rounded up by the stratified sampler), depth 5-8, RGB, seed 4")


def rank_jobs(paths: list[int], world: int) -> list[list[int]]:
    """Whole jobs per rank (no data-path collective): the largest job first,
    each to the rank with the fewest paths so far."""
    loads = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(paths)), key=lambda k: -paths[k]):
        r = min(range(world), key=lambda q: (loads[q], q))
        out[r].append(i)
        loads[r] += paths[i]
    return [sorted(x) for x in out]


def sample_desc(desc: dict, spp_actual: int, target: int) -> dict:
    """The job's scene with its screen edge cut so one pass renders at most
    about `target` paths at the job's own samples per pixel.  The projector's
    field of view (or extent) is kept, so the rays keep their distribution
    and every path costs what it costs in the full job."""
    import copy

    n = desc["n"]
    d = copy.deepcopy(desc)
    size = d["projector"]["size"]
    edge = max(2, min(size[0], int((target / spp_actual) ** (1.0 / (n - 1)))))
    if d["projector"]["type"] == "parallel":
        d["projector"]["units_per_pixel"] *= size[0] / edge
    d["projector"]["size"] = [edge] * (n - 1)
    return d


def _reference_job_worker(conn, desc: dict, spp: int, depth: int, passes: int, threads: int,
                          precision: str = "float", spectrum: bool = False, integrator: str = "bpt"):
    """Child process: the reference painter's scene once, then `passes`
    one-pass paints, each pass's (paths, seconds) sent as it ends."""
    from oracle import oracle

    s = oracle.Scene(desc, precision, spectrum)
    if integrator != "bpt":
        s.set_integrator(integrator)
    conn.send(("built", None))
    for _ in range(passes):
        st, _ = s.paint(spp, depth, passes=1, threads=threads)
        conn.send(("pass", (st["sample_count"], st["pass_duration"])))
    conn.close()


def reference_job_passes(desc: dict, spp: int, depth: int, passes: int, threads: int,
                         limit: float = 60.0, precision: str = "float", spectrum: bool = False,
                         integrator: str = "bpt") -> tuple[list, int]:
    """`passes` passes of the reference painter on one scene, in a child
    process.  The reference's painter can stop for good at the end of a
    pass: the thread that ends the last pass sets the stop flag
    (src/painter/painting/painting.cpp:113-115) while another thread that has
    left the first barrier may not have read it yet (:141-144); that thread
    then leaves without arriving at the second barrier (:161) and the others
    wait there forever.  Short passes make it likely.  A pass that does not
    end within `limit` seconds is abandoned: the child is killed and a new
    one renders the passes still to do.  Returns the passes' (paths, seconds)
    and the number of abandoned passes."""
    import multiprocessing

    ctx = multiprocessing.get_context("spawn")
    out: list = []
    hangs = 0
    while len(out) < passes:
        a, b = ctx.Pipe(duplex=False)
        p = ctx.Process(target=_reference_job_worker,
                        args=(b, desc, spp, depth, passes - len(out), threads, precision, spectrum, integrator),
                        daemon=True)
        p.start()
        b.close()
        ok = a.poll(1800.0)  # the scene build
        while ok and len(out) < passes:
            try:
                kind, v = a.recv()
            except EOFError:
                ok = False
                break
            if kind == "pass":
                out.append(v)
            if len(out) < passes:
                ok = a.poll(limit)
        if not ok:
            p.kill()
            hangs += 1
            print(f"reference painter: a pass did not end within {limit:.0f} s; restarted "
                  f"({len(out)} of {passes} passes done)", file=sys.stderr, flush=True)
            if hangs > 10:
                raise RuntimeError("the reference painter stopped at the end of a pass more than 10 times")
        p.join()
        a.close()
    return out, hangs


def reference_job_rates(jobs: list[dict], target: int, threads: int, steps: int = 1, warmup: int = 0) -> dict:
    """The reference's own painter (create_painter, float, RGB, all `threads`
    host threads, one job at a time) over a bounded sample of every job: the
    job's scene, samples per pixel and depth on a screen cut to about
    `target` paths (sample_desc).  `steps` timed steps (after `warmup`
    untimed ones) each render the next ceil(len(jobs) / steps) jobs one pass,
    so the timed steps cover every job.  Returns per-job paths/s and the
    batch's paths/s extrapolated to the full jobs: sum(paths) / sum(paths /
    rate)."""
    per_step = -(-len(jobs) // max(1, steps))
    timed = [0] * len(jobs)
    untimed = [0] * len(jobs)
    schedule = []
    for k in range(warmup + steps):
        group = [(k * per_step + m) % len(jobs) for m in range(per_step)]
        schedule.append(group)
        for g in group:
            (untimed if k < warmup else timed)[g] += 1
    rates = [None] * len(jobs)
    pass_seconds = [[] for _ in jobs]
    sampled = 0
    seconds = 0.0
    hangs = 0
    for k, j in enumerate(jobs):
        if timed[k] + untimed[k] == 0:
            continue
        aspp = j["paths"] // int(np.prod(j["desc"]["projector"]["size"]))
        out, h = reference_job_passes(sample_desc(j["desc"], aspp, target), j["spp"], j["max_depth"],
                                      untimed[k] + timed[k], threads)
        hangs += h
        print(f"reference painter: job {j['index']} done", file=sys.stderr, flush=True)
        kept = out[untimed[k]:]
        if kept:
            rates[k] = sum(p for p, _ in kept) / sum(t for _, t in kept)
            pass_seconds[k] = [t for _, t in kept]
            sampled += sum(p for p, _ in kept)
            seconds += sum(t for _, t in kept)
    full = sum(j["paths"] for j in jobs) / sum(j["paths"] / r for j, r in zip(jobs, rates))
    # seconds of each timed step: its jobs' passes
    used = [0] * len(jobs)
    step_seconds = []
    for group in schedule[warmup:]:
        t = 0.0
        for g in group:
            t += pass_seconds[g][used[g]]
            used[g] += 1
        step_seconds.append(t)
    return {"value": full, "job_rates": rates, "sampled_paths": sampled, "sampled_seconds": seconds,
            "abandoned_passes": hangs, "jobs_per_step": per_step, "step_seconds": step_seconds}


def batch_step(server, built: list, jobs: list[dict], seed: int = 1, read_images: bool = True) -> dict:
    """One step of the batch: every job one pass (its samples per pixel)
    through the job server, all submitted at once; the images read back.
    `span` is the device time from the first job's first kernel to the last
    job's last (CUDA events on the jobs' streams)."""
    ids = [server.submit_render(s, j["spp"], j["max_depth"], seed=seed, passes=1) for s, j in zip(built, jobs)]
    first, last = [], []
    totals = {"paths": 0, "launches": 0, "bytes": 0.0, "rays": 0, "nodes": 0, "facets": 0, "nonfinite": 0}
    images = []
    for s, i in zip(built, ids):
        info = server.wait(i)
        st = server.statistics(i)
        first.append(info["device_started"])
        last.append(info["device_finished"])
        size = record_bytes(s.n, s.precision)
        totals["paths"] += st["sample_count"]
        totals["launches"] += st["kernel_launches"] + 1  # + the images' resolve kernel
        totals["bytes"] += st["nodes"] * size["node"] + st["facets"] * size["facet"] + st["shapes"] * size["shape"]
        totals["rays"] += st["ray_count"]
        totals["nodes"] += st["nodes"]
        totals["facets"] += st["facets"]
        totals["nonfinite"] += st["nonfinite_samples"]
        if read_images:
            images.append(server.images(i, s.pixels)[0])
        server.release(i)
    totals["span"] = max(last) - min(first)
    totals["images"] = images
    return totals


def batch_steps(server, wave_scenes: list, waves: list, steps: int, seed: int = 1,
                read_images: bool = True) -> dict:
    """`steps` steps of the batch submitted back to back: step k renders
    wave k mod len(waves) (each job one pass at its own samples per pixel);
    all the steps' renders are queued in the job server at once, which
    admits them as slots and memory free up (continuous batching, no drain
    between steps).  `span` is the device time from the first job's first
    kernel to the last job's last (CUDA events on the jobs' streams);
    `images` holds each job's image of its last step."""
    work = [(s, j) for k in range(steps) for s, j in zip(wave_scenes[k % len(waves)], waves[k % len(waves)])]
    ids = [server.submit_render(s, j["spp"], j["max_depth"], seed=seed, passes=1) for s, j in work]
    first, last = [], []
    totals = {"paths": 0, "launches": 0, "bytes": 0.0, "rays": 0, "nodes": 0, "facets": 0, "nonfinite": 0}
    images = {}
    for (s, j), i in zip(work, ids):
        info = server.wait(i)
        st = server.statistics(i)
        first.append(info["device_started"])
        last.append(info["device_finished"])
        size = record_bytes(s.n, s.precision)
        totals["paths"] += st["sample_count"]
        totals["launches"] += st["kernel_launches"] + 1  # + the images' resolve kernel
        totals["bytes"] += st["nodes"] * size["node"] + st["facets"] * size["facet"] + st["shapes"] * size["shape"]
        totals["rays"] += st["ray_count"]
        totals["nodes"] += st["nodes"]
        totals["facets"] += st["facets"]
        totals["nonfinite"] += st["nonfinite_samples"]
        if read_images:
            images[j["index"]] = server.images(i, s.pixels)[0]
        server.release(i)
    totals["span"] = max(last) - min(first) if work else 0.0
    totals["images"] = images
    return totals


def e2e_step(server, jobs: list[dict], precision: str, builders: int = 4) -> dict:
    """One step of the batch end to end through the public API: every
    scene built from host arrays (nbpt_scene_* on `builders` host threads,
    each job submitted as soon as its scene is on the device), one pass per
    job through the job server, RGB and RGBA images read back."""
    from concurrent.futures import ThreadPoolExecutor

    from math_b200 import painter as P

    t0 = time.perf_counter()
    h2d = d2h = 0
    with ThreadPoolExecutor(builders) as ex:
        futures = [ex.submit(P.Scene, j["desc"], precision, False) for j in jobs]
        built, ids = [], []
        for f, j in zip(futures, jobs):
            s = f.result()
            built.append(s)
            ids.append(server.submit_render(s, j["spp"], j["max_depth"], seed=1, passes=1))
        for s, i in zip(built, ids):
            server.wait(i)
            rgb, rgba = server.images(i, s.pixels)
            d2h += rgb.nbytes + rgba.nbytes
            h2d += s.upload_bytes()
            server.release(i)
            s.close()
    return {"seconds": time.perf_counter() - t0, "h2d": h2d, "d2h": d2h}


def serve_stream(server, pool: list[dict], built: list, rate: float, duration: float, seed: int) -> dict:
    """Poisson arrivals of renders into the job server (continuous batching):
    each job draws a resident scene from the pool and a sample budget
    log-uniform in [16, 256] samples per pixel; the server creates the render
    when it admits the job.  Latency is completion minus arrival."""
    rng = np.random.default_rng(seed)
    arrivals = []
    t = 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        k = int(rng.integers(0, len(pool)))
        spp = int(round(math.exp(rng.uniform(math.log(16), math.log(256)))))
        # one pass renders at most 256 samples per pixel after the stratified
        # sampler rounds the count up to a power of the screen dimension
        while built[k].actual_spp(spp) > 256:
            spp -= 1
        arrivals.append((t, k, spp))
    t_start = server.time()
    submitted = []
    for a, k, spp in arrivals:
        while server.time() - t_start < a:
            time.sleep(min(0.001, max(0.0, a - (server.time() - t_start))))
        s = built[k]
        i = server.submit_render(s, spp, pool[k]["max_depth"], seed=len(submitted) + 1)
        submitted.append((i, t_start + a, s.pixels * s.actual_spp(spp)))
    latencies, waits = [], []
    last = t_start
    for i, arrival, _ in submitted:
        info = server.wait(i)
        latencies.append(info["finished"] - arrival)
        waits.append(info["started"] - arrival)
        last = max(last, info["finished"])
        server.release(i)
    paths = sum(p for _, _, p in submitted)
    lat = np.array(latencies) if latencies else np.zeros(1)
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_queue_wait_s": float(np.mean(waits)) if waits else 0.0, "jobs": len(submitted),
            "rate_per_s": rate, "duration_s": duration,
            "throughput_paths_per_second": paths / (last - t_start) if last > t_start else None,
            "offered_paths_per_second": paths / duration, "makespan_s": last - t_start}


def flush_l2(buf):
    import torch

    buf.fill_(1)
    torch.cuda.synchronize()


def run_batch(args, rank: int, world: int, local: int):
    import torch

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from math_b200 import painter as P
    from math_b200 import scenes

    workers = max(1, (os.cpu_count() or 1) // max(1, world))
    all_paths = scenes.mixed_batch_paths(args.jobs, BATCH_SEED, args.screen_scale)
    mine = rank_jobs(all_paths, world)[rank]
    t0 = time.perf_counter()
    jobs = scenes.mixed_batch(args.jobs, seed=BATCH_SEED, points_scale=args.points_scale,
                              screen_scale=args.screen_scale, workers=workers, select=mine)
    generate_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    fp32 = [P.Scene(j["desc"], "float", False) for j in jobs]
    build_s = time.perf_counter() - t0
    paths_per_batch = sum(j["paths"] for j in jobs)
    # the rank's jobs in waves of about equal paths; a step renders one wave
    groups = rank_jobs([j["paths"] for j in jobs], min(args.waves, len(jobs)))
    waves = [[jobs[k] for k in g] for g in groups]
    wave_scenes = [[fp32[k] for k in g] for g in groups]
    wave_paths = [sum(j["paths"] for j in w) for w in waves]
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    server = P.Server(max_jobs=args.max_jobs)
    try:
        tuning = None
        if args.tune:
            from math_b200 import tuning as T

            def one_batch():
                r = batch_steps(server, wave_scenes, waves, len(waves), read_images=False)
                return r["paths"], r["span"]

            # a first batch at the default allocates the scenes' buffers
            one_batch()
            # every candidate starts from an empty buffer cache, and so does
            # the warm-up after the tuning
            tuning = T.tune_chunk_budget(server, one_batch, T.chunk_budget_candidates(server),
                                         reset=P.release_cached_memory)
        server_chunk_budget = server.chunk_budget
        for k in range(args.warmup):
            flush_l2(flush)
            w = k % len(waves)
            batch_step(server, wave_scenes[w], waves[w], read_images=False)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        clocks = ClockSampler(local)
        clocks.start()
        spans = [[] for _ in waves]
        totals = {"launches": 0, "bytes": 0.0, "rays": 0, "nodes": 0, "facets": 0, "nonfinite": 0, "paths": 0}
        images = {}
        for k in range(args.steps):
            flush_l2(flush)
            w = k % len(waves)
            r = batch_step(server, wave_scenes[w], waves[w])
            spans[w].append(r["span"])
            for key in totals:
                totals[key] += r[key]
            for j, img in zip(waves[w], r["images"]):
                images[j["index"]] = img
        clock_info = clocks.stop()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        step_seconds = float(sum(sum(x) for x in spans))
        if all(spans):
            # every wave timed: the batch's rate from each wave's mean span
            # (the plain sum when the steps cover whole batches)
            rank_rate = paths_per_batch / sum(float(np.mean(x)) for x in spans)
        else:
            rank_rate = totals["paths"] / step_seconds
        # whole batch over the slowest rank: every rank renders its jobs
        batch_seconds = slowest_rank(paths_per_batch / rank_rate, world, "cuda")
        value = sum(all_paths) / batch_seconds

        # end to end through the public API: each wave's scenes from host
        # arrays, its jobs through the server, images back
        e2e_steps = max(1, args.e2e_steps if args.e2e_steps > 0 else len(waves))
        e2e = {"seconds": 0.0, "h2d": 0, "d2h": 0}
        e2e_paths = 0
        for k in range(e2e_steps):
            w = k % len(waves)
            r = e2e_step(server, waves[w], "float")
            e2e_paths += wave_paths[w]
            for key in e2e:
                e2e[key] += r[key]
        e2e_rate = e2e_paths / e2e["seconds"]
        e2e_value = sum(all_paths) / slowest_rank(paths_per_batch / e2e_rate, world, "cuda")

        plain = None
        serve = None
        if world == 1:
            plain = plain_fp64(args, jobs, paths_per_batch, [images.get(j["index"]) for j in jobs], flush)
            if args.serve_duration > 0:
                serve = serve_sub(args, server, workers, value)
    finally:
        server.close()

    if rank == 0:
        peaks = {}
        try:
            peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        except (OSError, ValueError):
            pass
        peak = peaks.get("hbm_gbs", 6650.0)
        achieved = totals["bytes"] / step_seconds / 1e9 if step_seconds > 0 else None
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            cpu = batch_cpu_baseline(args, jobs)
        dims = [j["desc"]["n"] for j in jobs]
        line = {
            "metric": "batched_fp32_paths_per_second", "value": value, "unit": "paths/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * step_seconds / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded generators)",
            "config": {"workload": BATCH_LABEL, "jobs": args.jobs, "jobs_this_rank": len(jobs),
                       "dims": {str(n): dims.count(n) for n in (3, 4, 5)}, "paths_per_batch": sum(all_paths),
                       "facets_max": max(scenes.describe(j["desc"])["facets"] for j in jobs),
                       "waves": len(waves), "wave_paths": wave_paths,
                       "step": (f"one wave: {len(jobs) // len(waves)} of the batch's jobs (the batch split into "
                                f"{len(waves)} waves of about equal paths), one pass each at its own samples "
                                "per pixel, all submitted to the job server at once, images read back; value = "
                                "paths of the whole batch / the sum of the waves' mean device spans"),
                       "max_jobs": args.max_jobs,
                       "chunk_budget": server_chunk_budget,
                       "tuning": tuning and {
                           "what": "the job server's chunk budget per render, chosen before the warm-up by "
                                   "math_b200.tuning: one batch per candidate, the fastest kept",
                           "chosen_gib": tuning["chosen"] / 2**30,
                           "trials": [{"chunk_budget_gib": t["chunk_budget"] / 2**30,
                                       "paths_per_s": t["paths_per_s"]} for t in tuning["trials"]]},
                       "points_scale": args.points_scale,
                       "screen_scale": args.screen_scale, "generate_s": generate_s, "scene_build_s": build_s,
                       "l2": "flushed (256 MiB write) before every step; scenes and buffers exceed L2",
                       "timing": "device span per step: CUDA events on the jobs' streams, from the first kernel of "
                                 "the wave's first job to the last kernel of its last job"},
            "plain_fp64": plain,
            "speedup_vs_plain_fp64": (value / plain["value"]) if plain else None,
            "e2e": {"value": e2e_value, "unit": "paths/s",
                    "h2d_bytes_per_step": int(e2e["h2d"] / e2e_steps), "d2h_bytes_per_step": int(e2e["d2h"] / e2e_steps),
                    "steps": e2e_steps, "seconds": e2e["seconds"],
                    "note": "every step one wave through the C ABI: each scene built from host arrays (mesh "
                            "ingestion, host->device copies, BVH build and facet setup on the GPU) on 4 host threads "
                            "and submitted when ready, one pass per job, RGB and RGBA images read back; host clock"},
            "serve": serve,
            "gpu_launches": totals["launches"],
            "nonfinite_samples": totals["nonfinite"],
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": None,
                         "kernel": "whole steps: path kernels, estimator and resolve of all jobs, overlapped across "
                                   "jobs (algorithmic scene bytes counted on the device / device span)",
                         "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                         "algorithmic_bytes_per_path": totals["bytes"] / totals["paths"],
                         "node_visits_per_path": totals["nodes"] / totals["paths"],
                         "facet_tests_per_path": totals["facets"] / totals["paths"],
                         "rays_per_path": totals["rays"] / totals["paths"]},
            "clocks": clock_info,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def plain_fp64(args, jobs, paths_per_step, fp32_images, flush) -> dict:
    """The plain comparator: the same jobs in FP64, one at a time (a job
    server with one slot), the same kernels; one warm-up job per dimension,
    then one timed batch."""
    from math_b200 import painter as P

    t0 = time.perf_counter()
    fp64 = [P.Scene(j["desc"], "double", False) for j in jobs]
    build_s = time.perf_counter() - t0
    one = P.Server(max_jobs=1)
    try:
        seen = set()
        for s, j in zip(fp64, jobs):
            if j["desc"]["n"] not in seen:
                seen.add(j["desc"]["n"])
                batch_step(one, [s], [j], read_images=False)
        flush_l2(flush)
        w0 = time.perf_counter()
        r = batch_step(one, fp64, jobs)
        wall = time.perf_counter() - w0
    finally:
        one.close()
    rmse = [rel_rmse(a, b) for a, b in zip(fp32_images or [], r["images"]) if a is not None]
    for s in fp64:
        s.close()
    return {"value": paths_per_step / r["span"], "seconds": r["span"], "wall_seconds": wall,
            "scene_build_s": build_s, "steps": 1,
            "note": "FP64 scenes, one job at a time through a job server with one slot (painter created at "
                    "admission, one pass, images read back), device span as for value",
            "same_seed_rel_rmse_fp32_vs_fp64": {
                "median": float(np.median(rmse)) if rmse else None, "max": float(np.max(rmse)) if rmse else None,
                "note": "one pass each on the same streams: float rounding moves paths off their double twins, "
                        "so this is per-pass sample noise, not bias (bias against converged FP64 images is in "
                        "tests/test_config_parity.py)"}}


def serve_sub(args, server, workers: int, capacity: float) -> dict:
    """Served stream beside the batch: Poisson arrivals at a rate that offers
    `serve_load` of the measured batched throughput (the stated 40 jobs/s
    offers about 30 times what one B200 renders, so its queue only grows)."""
    from math_b200 import painter as P
    from math_b200 import scenes

    pool = scenes.mixed_batch(args.pool, seed=SERVE_SEED, workers=workers)
    built = [P.Scene(j["desc"], "float", False) for j in pool]
    # mean paths per job of the arrival mix: pool scene x spp log-uniform [16, 256]
    sizes = []
    for s, j in zip(built, pool):
        sp = [min(256, s.actual_spp(int(round(math.exp(x))))) for x in np.linspace(math.log(16), math.log(256), 9)]
        sizes.append(s.pixels * float(np.mean(sp)))
    mean_paths = float(np.mean(sizes))
    rate = args.serve_load * capacity / mean_paths
    for s, j in zip(built, pool):  # warm-up: one small render of every pool scene
        i = server.submit_render(s, 4, j["max_depth"], seed=1)
        server.wait(i)
        server.release(i)
    out = serve_stream(server, pool, built, rate, args.serve_duration, SERVE_SEED)
    out["offered_load"] = args.serve_load
    out["note"] = (f"Poisson arrivals for {args.serve_duration:.0f} s at {rate:.2f} jobs/s, offering "
                   f"{args.serve_load:.0%} of the measured batched throughput; scenes drawn as in the batch "
                   f"(seed {SERVE_SEED}, a resident pool of {args.pool}), 16-256 spp log-uniform.  The stated 40 "
                   "jobs/s offers about 30x what one B200 renders: its queue grows without bound and p99 is set "
                   "by the stream's length")
    for s in built:
        s.close()
    return out


def batch_cpu_baseline(args, jobs) -> dict:
    """The reference painter on the host cores over a bounded sample of the
    batch: every fourth job, one pass each on a screen cut to about
    --ref-target paths."""
    from oracle import oracle

    if not oracle.available():
        return {"value": None, "unit": "paths/s", "cores": 0, "kind": "reference",
                "sample": "oracle library not built"}
    subset = jobs[::4]
    cores = os.cpu_count() or 1
    r = reference_job_rates(subset, args.ref_target, cores, steps=1)
    return {"value": r["value"], "unit": "paths/s", "cores": cores, "kind": "reference",
            "sample": (f"the reference's create_painter (float, RGB, {cores} threads) on {len(subset)} of the "
                       f"{len(jobs)} jobs (every fourth), one pass each, each job's scene, samples per pixel and depth "
                       f"on a screen cut to about {args.ref_target} paths; {r['sampled_paths']} paths in "
                       f"{r['sampled_seconds']:.1f} s; value = sum(paths) / sum(paths / job rate) over those jobs "
                       "at full size")}


def run_reference_batch(args, rank: int):
    """--impl reference on the batch: the reference's own CPU painter, one
    job at a time, every job of the batch each step on a bounded sample."""
    if rank != 0:
        return
    from math_b200 import scenes
    from oracle import oracle

    if not oracle.available():
        print(json.dumps({"impl": "reference", "unavailable": "the reference painter (oracle/_ref) is not built"}))
        return
    cores = os.cpu_count() or 1
    jobs = scenes.mixed_batch(args.jobs, seed=BATCH_SEED, points_scale=args.points_scale,
                              screen_scale=args.screen_scale, workers=cores)
    r = reference_job_rates(jobs, args.ref_target, cores, steps=args.steps, warmup=args.warmup)
    value = r["value"]
    paths = sum(j["paths"] for j in jobs)
    sample = (f"each step: the reference's create_painter (float, RGB, {cores} threads) on the next "
              f"{r['jobs_per_step']} of the {len(jobs)} jobs (the timed steps cover every job), one at a time, each "
              f"job's scene, samples per pixel and depth on a screen cut to about {args.ref_target} paths; value = "
              f"sum(paths) / sum(paths / job rate) over the full jobs ({r['sampled_paths']} paths sampled in "
              f"{r['sampled_seconds']:.1f} s; {r['abandoned_passes']} passes abandoned to the painter's end-of-pass "
              "stop race and rendered again)")
    print(json.dumps({
        "metric": "batched_fp32_paths_per_second", "value": value, "unit": "paths/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * float(np.mean(r["step_seconds"])), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators)",
        "config": {"workload": BATCH_LABEL, "jobs": args.jobs, "paths_per_batch": paths,
                   "seconds_per_batch_extrapolated": paths / value},
        "cpu_baseline": {"value": value, "unit": "paths/s", "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "paths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_serve(args):
    """Poisson arrivals of renders into the job server at --rate jobs/s for
    --duration s (C5 as stated: 40 jobs/s), with completion latencies."""
    from math_b200 import painter as P
    from math_b200 import scenes

    pool = scenes.mixed_batch(args.pool, seed=SERVE_SEED, points_scale=args.points_scale,
                              screen_scale=args.screen_scale, workers=os.cpu_count() or 1)
    built = [P.Scene(j["desc"], "float", False) for j in pool]
    server = P.Server(max_jobs=args.max_jobs)
    try:
        for s, j in zip(built, pool):
            i = server.submit_render(s, 4, j["max_depth"], seed=1)
            server.wait(i)
            server.release(i)
        out = serve_stream(server, pool, built, args.rate, args.duration, SERVE_SEED)
    finally:
        server.close()
    line = {"metric": "served_job_latency_p99", "value": out["p99_s"], "unit": "s", "higher_is_better": False,
            "n_gpus": 1, **out, "dtype": "f32", "data": "synthetic (seeded generators)",
            "config": {"workload": "Poisson render arrivals into the job server", "rate_per_s": args.rate,
                       "duration_s": args.duration, "pool_scenes": len(pool), "spp": "log-uniform 16-256",
                       "max_jobs": args.max_jobs}}
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
        if args.workload == "batch":
            run_reference_batch(args, rank)
        else:
            run_reference(args, rank)
        return
    if args.workload == "batch":
        run_batch(args, rank, world, local)
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
