#!/usr/bin/env python
"""Throughput of the collision/contact pipeline on B200, in body-steps/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload c4|c2|c3|c5]

Workloads (seeded synthetic scenes, ag2d.scenes):
  c4 (default)  4,096 independent worlds, body counts log-uniform in [16, 2048] (c1 mix: 3-8-gons on a ground box),
                packed into one batch and advanced by one launch sequence per step; the same worlds stepped one
                world per launch sequence are timed beside it ("per_world_launch").
  c2            one world of 100,000 mixed bodies dropped into a static U container.
  c3            1,000,000 circles and 4-6-gons: collision detection alone (poses, AABBs, Morton, sort, LBVH,
                query, SAT), reported as broad+narrow GB/s against the HBM roofline, with the exact pair count
                checked against the oracle's sweep.
  c5            serving: requests arrive as a Poisson stream (lambda 2,000/s), each a world of log-uniform
                [32, 8192] bodies (c1 mix, 5% small fast circles, continuous collision detection on) asking for 120
                steps, admitted against a 120 GB budget into one resident batch (ag2d.Server); a fixed-length run of
                --requests arrivals, reporting aggregate body-steps/s and p50 / p99 completion latency.

One process per GPU (torchrun for N > 1). Worlds exchange nothing on the step path, so each rank advances its own
batch: the job's N x 4,096 worlds (seeds 0 ..) are shared out by greedy body-count balancing (largest first, to the
least-loaded rank): weak scaling with no collective in the step; the whole-job value is the sum of all ranks'
body-steps over the slowest rank's device time.

Timing: c4 steps every world from rest to --window-start - W, then W untimed warm-up steps, then K timed steps
(both arms time the same window), each bracketed by CUDA events on the engine's stream, with a 256 MiB write
between steps outside the events (L2 flushed); barrier + synchronize around the timed region; the max over ranks.
SM clocks are sampled with nvidia-smi during the timed region. The end-to-end number ("e2e") goes through the C ABI
with host buffers: a page-locked host checkpoint of the window's start is loaded into a resident engine inside the
timed region (ag2d_batch_load; the engine was allocated before it, as a server's is), then per step one step call
and one asynchronous read of every body's pose into page-locked host memory, waited for one step later.

--impl reference times the reference engine itself (oracle/_ref/libagony_ref.so, its own C++ on the host cores,
all threads) on a bounded sample of the same workload and prints the same line with "impl": "reference".
"""
from __future__ import annotations

import argparse
import json
import os
import queue
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "physicssimulation-agony_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "body-steps/s"
WORKLOADS = {
    "c4": "c4: 4096 independent worlds, body counts log-uniform [16, 2048] (3-8-gons r U[0.5,2] +-15% jitter on a "
          "static 220 m ground box each), dt 1/60, 8 velocity + 3 position iterations, batched",
    "c2": "c2: single large world, 100k mixed bodies (60% boxes, 25% circles, 15% 3-8-gons) in a static U, "
          "dt 1/60, 8 velocity + 3 position iterations, stepped from the drop",
    "c3": "c3: 1M bodies (50% circles, 50% 4-6-gons, size log-uniform 0.1-2 m) uniform in 4000 x 4000 m, "
          "v ~ N(0, 5 m/s); collision detection alone (poses, AABBs, Morton, sort, LBVH, query, SAT)",
    "c5": "c5: serving, Poisson arrivals at 2000 req/s, each a world of log-uniform [32, 8192] bodies (c1 mix, 5% "
          "circles r 0.05 m at 200 m/s, CCD on) for 120 steps, 120 GB admission budget, continuous batching",
}
DEFAULT_STEPS = {"c4": 600, "c2": 1000, "c3": 20, "c5": 120}
BODY_UPLOAD_BYTES = 16 + 16 + 8 + 4 + 4 + 4 + 1 + 4 + 4 + 4 + 4 + 16   # body + collider records as uploaded


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c4", choices=sorted(WORKLOADS))
    ap.add_argument("--worlds", type=int, default=4096)
    ap.add_argument("--bodies", type=int, default=None, help="c2 / c3 body count")
    ap.add_argument("--per-world-sample", type=int, default=256)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-autotune", action="store_true",
                    help="c4: keep the engine's default launch shapes (shorter runs, e.g. under a profiler)")
    ap.add_argument("--tune-ahead", type=int, default=300,
                    help="c4: steps a copy of the batch runs before the autotuner times launch shapes on it")
    ap.add_argument("--requests", type=int, default=4000, help="c5 arrivals in the timed run")
    ap.add_argument("--rate", type=float, default=2000.0, help="c5 Poisson arrival rate, requests/s")
    ap.add_argument("--budget-gb", type=float, default=120.0, help="c5 admission budget")
    ap.add_argument("--round-steps", type=int, default=8, help="c5 steps between admission rounds")
    ap.add_argument("--reserve-bodies", type=int, default=4_000_000,
                    help="c5 resident bodies the server sizes its batch for at start-up")
    ap.add_argument("--window-start", type=int, default=300,
                    help="c4: first step of the timed window (both arms step every world from rest to it)")
    ap.add_argument("--no-extras", action="store_true",
                    help="c4: leave out the c3 collision-detection and c5 serving sub-results of the default line")
    ap.add_argument("--extra-requests", type=int, default=2000, help="c5 arrivals of the default line's c5 part")
    ap.add_argument("--checkpoint", default=None,
                    help="c4: file (per rank: PATH.rankR) holding the batch at step window-start - warmup: written "
                         "after settling when missing, restored instead of settling when present (profiler runs)")
    a = ap.parse_args()
    if a.window_start < a.warmup:
        ap.error("--window-start must be at least --warmup")
    if a.steps is None:
        a.steps = DEFAULT_STEPS[a.workload]
    if a.bodies is None:
        a.bodies = 1_000_000 if a.workload == "c3" else 100_000
    return a


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------------------------------------------
# Scenes
# ---------------------------------------------------------------------------------------------------------------
def c4_shard(worlds_per_rank, rank, world_size):
    """This rank's worlds of the whole job (worlds_per_rank x world_size worlds, seed 0), balanced by body count
    over the ranks (weak scaling: the per-rank load stays at one batch's worth)."""
    from ag2d import scenes
    counts = scenes.c4_counts(worlds_per_rank * world_size, 0)
    return scenes.shard_by_bodies(counts, world_size)[rank]


def c4_scenes(worlds, seed=0, rank=0, world_size=1):
    from ag2d import scenes
    subset = None if world_size == 1 else c4_shard(worlds, rank, world_size)
    return scenes.make_c4_worlds(worlds=worlds * world_size, seed=seed, processes=max(1, min(32, host_threads())),
                                 subset=subset)


def c5_requests(count, seed):
    from ag2d import scenes
    return scenes.make_c5_requests(count, seed=seed, processes=max(1, min(32, host_threads())))


def poisson_arrivals(count, rate, seed):
    import numpy as np
    return np.cumsum(np.random.default_rng(seed ^ 0xA221).exponential(1.0 / rate, count))


def c2_scene(n):
    from ag2d import scenes
    cols = 500 if n >= 100_000 else max(10, int(round((n / 200.0) ** 0.5 * 10)))
    return scenes.make_c2(n, 0, columns=cols)


def c3_scene(n):
    from ag2d import scenes
    return scenes.make_c3(n, 0, extent=4000.0 * (n / 1e6) ** 0.5)


def mean_shape_bytes(scene_list):
    import numpy as np
    from ag2d import roofline, scenes
    total, count = 0.0, 0
    for sc in scene_list:
        k = sc.kind.astype(np.int64)
        total += float(np.where(k == scenes.POLYGON, 8.0 + 16.0 * sc.poly_count,
                                np.where(k == scenes.BOX, roofline.SHAPE_BYTES[1], roofline.SHAPE_BYTES[0])).sum())
        count += sc.n
    return total / max(count, 1)


def upload_bytes(scene_list):
    return sum(sc.n * BODY_UPLOAD_BYTES + int(sc.poly_count.sum()) * 16 for sc in scene_list)


# ---------------------------------------------------------------------------------------------------------------
# Measurement helpers
# ---------------------------------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi sampled every 200 ms while running (the clocks line of the timing rules)."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        # nvidia-smi's start-up (driver and NVML initialisation over every GPU of the node) can hold the driver
        # for a few hundred milliseconds: wait for its first sample so that it is done before the timed region.
        deadline = time.perf_counter() + 10.0
        while time.perf_counter() < deadline and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.02)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except OSError:
            rows = []
        finally:
            if self.path and os.path.exists(self.path):
                os.unlink(self.path)
        clk, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                clk.append(float(r[1]))
                mx.append(float(r[2]))
                for k, name in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        if clk:
            out = {"sm_mhz": statistics.median(clk), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                   "samples": len(clk)}
        return out


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def dram_traffic(kernel):
    """Per-launch DRAM bytes of a kernel (for the bench's workload) from the committed ncu summary, or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic.json")) as f:
            return json.load(f).get(kernel)
    except (OSError, ValueError):
        return None


class Timer:
    """Per-step device time on one stream: CUDA events around each step, an L2 flush between steps."""

    def __init__(self, torch, stream, dev):
        self.torch = torch
        self.stream = stream
        self.flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)   # 256 MiB > 126 MB L2
        self.ms = []

    def run(self, fn, steps, on_step=None):
        torch = self.torch
        for _ in range(steps):
            with torch.cuda.stream(self.stream):
                self.flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(self.stream)
            fn()
            e1.record(self.stream)
            e1.synchronize()
            self.ms.append(e0.elapsed_time(e1))
            if on_step:
                on_step()
        return float(sum(self.ms))


def roofline_line(phases, bytes_by_phase, kernel_of, workload, solve_passes=None):
    """The dominant phase's roofline. For the solver, solve_passes (bytes by pass, whole run) is listed per launch
    beside the total, with the velocity passes' own fraction (the measurement unit's 192 B per manifold per
    velocity iteration over the whole kernel's time, a lower bound on what those passes reach)."""
    dominant = max(bytes_by_phase, key=lambda p: phases[p][0])
    peak, peak_kind = measured_peaks()
    dom_ms, dom_calls = phases[dominant]
    achieved = bytes_by_phase[dominant] / max(dom_ms / 1e3, 1e-12) / 1e9
    calls = max(dom_calls, 1)
    traffic = dram_traffic(f"{workload}:{kernel_of[dominant]}")
    line = {"bound": "hbm", "kernel": kernel_of[dominant], "phase": dominant, "achieved": achieved, "peak": peak,
            "unit": "GB/s", "frac": achieved / peak, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
            "traffic": traffic, "algorithmic_bytes_per_launch": bytes_by_phase[dominant] / calls,
            "launch_ms": dom_ms / calls}
    if traffic:
        line["traffic_frac"] = traffic / max(dom_ms / calls / 1e3, 1e-12) / 1e9 / peak   # measured DRAM bytes
    if dominant == "solve" and solve_passes:
        line["bytes_per_launch_by_pass"] = {k: v / calls for k, v in solve_passes.items()}
        line["velocity_passes_frac"] = solve_passes["velocity"] / max(dom_ms / 1e3, 1e-12) / 1e9 / peak
    return line


def solve_passes(manifolds_sum, vi=8, pi=3):
    from ag2d import roofline
    return roofline.solve_bytes_breakdown(manifolds_sum, vi, pi)


def step_bytes(msb, pairs_sum, manifolds_sum, dyn_bodies, steps, vi=8, pi=3):
    from ag2d import roofline
    K = steps
    return {
        "solve": roofline.solve_bytes(manifolds_sum, vi, pi),
        "narrow": roofline.narrow_bytes(pairs_sum, msb, manifolds_sum),
        "integrate": roofline.integrate_bytes(dyn_bodies * K),
        "pose": roofline.pose_bytes(dyn_bodies * K, msb),
        "sort": roofline.sort_bytes(dyn_bodies * K),
        "query": roofline.query_bytes(dyn_bodies * K, pairs_sum),
    }


def diagnostics(c0, c1, per_step, colors_sum, K):
    return {"mean_colors": colors_sum / K, "list_rebuilds": c1["list_rebuilds"] - c0["list_rebuilds"],
            "retries": c1["retries"] - c0["retries"], "regrows": c1["regrows"] - c0["regrows"],
            "device_allocs": c1["device_allocs"] - c0["device_allocs"],
            "host_ms_per_step": (c1["host_ms"] - c0["host_ms"]) / K,
            "sync_wait_ms_per_step": (c1["sync_ms"] - c0["sync_ms"]) / K,
            "max_step_ms": max(per_step), "max_step_index": per_step.index(max(per_step)),
            "median_step_ms": statistics.median(per_step)}


def reduce_max(torch, dist, world_size, dev, value):
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    if world_size > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(torch, dist, world_size, dev, value):
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    if world_size > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_rate(torch, dist, world_size, dev, units, seconds):
    """Whole-job rate: the units all ranks processed over the slowest rank's time. Returns (rate, slowest seconds,
    total units)."""
    slowest = reduce_max(torch, dist, world_size, dev, seconds)
    total = reduce_sum(torch, dist, world_size, dev, float(units))
    return total / slowest, slowest, total


def rank_seed(rank, per_rank):
    """First seed of a rank's worlds or requests: ranks draw disjoint seed ranges."""
    return rank * per_rank


# ---------------------------------------------------------------------------------------------------------------
# CPU baselines: the reference engine (oracle/_ref) on the host cores
# ---------------------------------------------------------------------------------------------------------------
def cpu_worlds_rate(scene_list, seconds, threads, max_steps=600, ccd=False):
    """Reference Simulation objects, one world per task, over a pool of host threads (ctypes releases the GIL).
    Each task creates its world and steps it in chunks of 10 until max_steps or the time budget; body-steps/s."""
    from oracle import refapi
    work = queue.Queue()
    for sc in scene_list:
        work.put(sc)
    done = [0.0]
    lock = threading.Lock()
    deadline = time.perf_counter() + seconds

    def worker():
        while time.perf_counter() < deadline:
            try:
                sc = work.get_nowait()
            except queue.Empty:
                return
            sim = refapi.RefSim(sc, threads=0, ccd=ccd)
            steps = 0
            while time.perf_counter() < deadline and steps < max_steps:
                sim.update(10)
                steps += 10
            sim.close()
            with lock:
                done[0] += sc.n * steps
    t0 = time.perf_counter()
    pool = [threading.Thread(target=worker) for _ in range(threads)]
    for t in pool:
        t.start()
    for t in pool:
        t.join()
    return done[0] / (time.perf_counter() - t0)


def cpu_worlds_window(scene_list, start, steps, threads, single_thread_worlds=0):
    """The reference engine over the step window [start, start + steps) of each world, on a pool of host threads
    (ctypes releases the GIL): every world is built and stepped to `start` untimed, then, after all are there, the
    pool steps every world through the window and the wall clock of that phase alone is the time. Returns
    (body-steps/s with `threads` threads, body-steps/s of one thread over the first `single_thread_worlds` worlds
    or None)."""
    from oracle import refapi
    settled = []
    lock = threading.Lock()
    work = queue.Queue()
    for sc in scene_list:
        work.put(sc)

    def settle():
        while True:
            try:
                sc = work.get_nowait()
            except queue.Empty:
                return
            sim = refapi.RefSim(sc, threads=0)
            sim.update(start)
            with lock:
                settled.append((sc.n, sim))
    pool = [threading.Thread(target=settle) for _ in range(threads)]
    for t in pool:
        t.start()
    for t in pool:
        t.join()
    one = None
    if single_thread_worlds:
        # One thread, one world after another, over the window (these worlds are then past it: timed first).
        sub = settled[:single_thread_worlds]
        t0 = time.perf_counter()
        for _, sim in sub:
            sim.update(steps)
        one = sum(n for n, _ in sub) * steps / (time.perf_counter() - t0)
        settled = settled[single_thread_worlds:]
    for item in settled:
        work.put(item)

    def run():
        while True:
            try:
                _, sim = work.get_nowait()
            except queue.Empty:
                return
            sim.update(steps)
    pool = [threading.Thread(target=run) for _ in range(threads)]
    t0 = time.perf_counter()
    for t in pool:
        t.start()
    for t in pool:
        t.join()
    elapsed = time.perf_counter() - t0
    for _, sim in settled:
        sim.close()
    return sum(n for n, _ in settled) * steps / elapsed, one


def c4_cpu_sample(scene_list):
    """Every 4th world of the batch (about a quarter of its bodies, the same size mix)."""
    stride = 4 if len(scene_list) >= 64 else 1
    return scene_list[::stride], stride


def cpu_c4(scene_list, start, steps):
    from oracle import refapi
    if not refapi.available():
        return None
    threads = host_threads()
    sample, stride = c4_cpu_sample(scene_list)
    one_worlds = min(64, len(sample) // 4)
    value, one = cpu_worlds_window(sample, start, steps, threads, one_worlds)
    return {"value": value, "unit": METRIC, "cores": threads, "kind": "reference",
            "sample": f"reference engine (oracle/_ref, -O2 -mavx2 -mfma), one single-threaded Simulation per world, "
                      f"every {stride}-th world of the batch ({len(sample)} worlds), each stepped to step {start} "
                      f"untimed, then steps {start}..{start + steps} timed on {threads} host threads (wall clock of "
                      f"that phase)",
            "single_thread": {"value": one, "cores": 1,
                              "sample": f"the first {one_worlds} of those worlds one after another on one thread, "
                                        f"same window"}}


def cpu_c2(scene, seconds):
    from oracle import refapi
    if not refapi.available():
        return None
    threads = max(0, host_threads() - 1)
    sim = refapi.RefSim(scene, threads=threads)
    steps, elapsed = 0, 0.0
    while elapsed < seconds and steps < 100000:
        elapsed += sim.timed_update(1)
        steps += 1
    sim.close()
    return {"value": scene.n * steps / elapsed, "unit": METRIC, "cores": threads + 1, "kind": "reference",
            "sample": f"reference engine (oracle/_ref, -O2 -mavx2 -mfma) on the first {steps} steps of the same "
                      f"{scene.n}-body world from the drop, {threads + 1} threads, {elapsed:.1f} s wall"}


def cpu_c3(scene, reps):
    from oracle import refapi
    if not refapi.available():
        return None
    threads = max(0, host_threads() - 1)
    sim = refapi.RefSim(scene, threads=threads)
    sim.timed_collide()
    times, pairs, mans = [], 0, 0
    for _ in range(reps):
        t, pairs, mans = sim.timed_collide()
        times.append(t)
    sim.close()
    return {"seconds": statistics.median(times), "pairs": pairs, "manifolds": mans, "threads": threads + 1}


def window_name(args):
    return f"steps {args.window_start}..{args.window_start + args.steps} of every world (stepped from rest)"


def reference_c3_extra(args):
    """The reference's collision-detection pass over the c3 world (the c3 line's CPU number)."""
    scene = c3_scene(1_000_000)
    r = cpu_c3(scene, 3)
    from ag2d import roofline
    step_b = roofline.broad_narrow_bytes_per_step(scene.n, mean_shape_bytes([scene]), r["pairs"], r["manifolds"])
    return {"workload": WORKLOADS["c3"], "value": scene.n / r["seconds"], "unit": METRIC,
            "ms_per_pass": 1e3 * r["seconds"], "pairs": r["pairs"], "manifolds": r["manifolds"],
            "broadphase_gbs": step_b / r["seconds"] / 1e9, "cores": r["threads"],
            "sample": "median of 3 collision-detection passes (spatial data, broad, narrow; agref_timed_collide)"}


def reference_c5_extra(args):
    """The reference serving c5 requests: a pool of host threads, one single-threaded Simulation per request."""
    scene_list = c5_requests(256, 0)
    threads = host_threads()
    seconds = 15.0
    value = cpu_worlds_rate(scene_list, seconds, threads, max_steps=120, ccd=True)
    return {"workload": WORKLOADS["c5"], "value": value, "unit": METRIC, "cores": threads,
            "sample": f"the first {len(scene_list)} requests of the stream, one single-threaded Simulation each "
                      f"(CCD on), {threads} at a time, 120 steps each, {seconds:.0f} s of serving; arrivals are not "
                      f"replayed on the host, so no latency"}


# ---------------------------------------------------------------------------------------------------------------
# Reference arm
# ---------------------------------------------------------------------------------------------------------------
def run_reference(args):
    rank, _, _ = dist_env()
    if rank != 0:
        return
    from oracle import refapi
    if not refapi.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libagony_ref.so was not built"}))
        return
    budget = 150.0
    base = {"impl": "reference", "metric": METRIC, "unit": METRIC, "n_gpus": 0, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
            "data": "synthetic (seeded scene generator, ag2d.scenes)"}
    if args.workload == "c4":
        scene_list = c4_scenes(args.worlds, 0)
        r = cpu_c4(scene_list, args.window_start, args.steps)
        value, threads, sample = r["value"], r["cores"], r["sample"]
        bodies = int(sum(s.n for s in scene_list))
        line = dict(base, value=value, steps=args.steps, ms_per_step=1e3 * bodies / value,
                    config={"workload": WORKLOADS["c4"], "worlds": args.worlds, "bodies": bodies,
                            "window": window_name(args),
                            "ms_per_step": "equivalent time of one step of the whole batch at this rate"},
                    single_thread=r["single_thread"])
        if not args.no_extras:
            line["c3"] = reference_c3_extra(args)
            line["c5"] = reference_c5_extra(args)
    elif args.workload == "c2":
        scene = c2_scene(args.bodies)
        threads = max(0, host_threads() - 1)
        sim = refapi.RefSim(scene, threads=threads)
        sim.update(args.warmup)
        steps, elapsed = 0, 0.0
        while steps < args.steps and elapsed < budget:
            elapsed += sim.timed_update(1)
            steps += 1
        sim.close()
        value = scene.n * steps / elapsed
        threads += 1
        sample = f"steps {args.warmup}..{args.warmup + steps} of the {scene.n}-body world ({threads} threads)"
        if steps < args.steps:
            sample += f"; stopped after {budget:.0f} s of {args.steps} requested steps"
        line = dict(base, value=value, steps=steps, ms_per_step=1e3 * elapsed / max(steps, 1),
                    config={"workload": WORKLOADS["c2"], "bodies": scene.n})
    elif args.workload == "c5":
        # The reference serves a request by stepping its own Simulation: requests are served by a pool of host
        # threads, one single-threaded Simulation each, 120 steps, over a bounded sample of the stream.
        scene_list = c5_requests(min(args.requests, 512), 0)
        threads = host_threads()
        seconds = min(budget, 30.0)
        value = cpu_worlds_rate(scene_list, seconds, threads, max_steps=args.steps, ccd=True)
        sample = (f"the first {len(scene_list)} requests of the stream, one single-threaded Simulation each (CCD "
                  f"on), {threads} at a time, {args.steps} steps each, {seconds:.0f} s of serving")
        line = dict(base, value=value, steps=args.steps, ms_per_step=None,
                    config={"workload": WORKLOADS["c5"], "requests": len(scene_list),
                            "note": "throughput of the host pool; arrivals are not replayed on the host"})
    else:
        scene = c3_scene(args.bodies)
        r = cpu_c3(scene, max(1, min(args.steps, 5)))
        threads = r["threads"]
        value = scene.n / r["seconds"]
        sample = f"median of collision-detection passes over the {scene.n}-body world ({threads} threads)"
        line = dict(base, value=value, steps=1, ms_per_step=1e3 * r["seconds"],
                    config={"workload": WORKLOADS["c3"], "bodies": scene.n, "pairs": r["pairs"]})
    line["cpu_baseline"] = {"value": value, "unit": METRIC, "cores": threads, "kind": "reference", "sample": sample}
    line["e2e"] = {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    print(json.dumps(line))


# ---------------------------------------------------------------------------------------------------------------
# Our arm
# ---------------------------------------------------------------------------------------------------------------
def run_c4(args, torch, dist, rank, world_size, local, dev):
    import ag2d
    scene_list = c4_scenes(args.worlds, 0, rank, world_size)
    n_bodies = int(sum(s.n for s in scene_list))
    settings = dict(dt=scene_list[0].dt, velocity_iterations=8, position_iterations=3, gravity=scene_list[0].gravity,
                    device=local)
    start, W, K = args.window_start, args.warmup, args.steps
    ckpt_file = f"{args.checkpoint}.rank{rank}" if args.checkpoint else None
    worlds = []
    if ckpt_file and os.path.exists(ckpt_file):
        # The settled state saved by an earlier run with the same arguments (step start - W of every world).
        raw = np.fromfile(ckpt_file, dtype=np.uint8)
        blob = ag2d.host_empty(raw.nbytes)
        blob[:] = raw
        batch = ag2d.Batch.restore(blob, device=local)
        del raw, blob
    else:
        for sc in scene_list:   # host objects only: a world touches the device on its first step
            w = ag2d.World(**settings)
            w.add_scene(sc)
            worlds.append(w)
        batch = ag2d.Batch(worlds)
        # Untimed: the batch steps from rest to the window's start (the reference arm steps the same worlds the
        # same way). Launch shapes are tuned on a copy restored from a checkpoint there; results do not depend on
        # them.
        batch.step(start - W)
        if ckpt_file:
            batch.save().tofile(ckpt_file)
    e = batch.engine
    stream = torch.cuda.ExternalStream(e.stream(), device=dev)
    if args.no_autotune:
        tuning = None   # the engine's default launch shapes (the settled-state choice on this workload)
    else:
        ahead = ag2d.Batch.restore(batch.save())
        tuning = ahead.engine.autotune(2)
        ahead.close()
        del ahead
        e.set_tuning(tuning)
    batch.step(W)
    ckpt = batch.save()   # host checkpoint at the window's start, for the end-to-end run below
    e.set_profiling(True)
    c0 = e.counters()
    if world_size > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sums = {"pairs": 0, "manifolds": 0, "colors": 0}

    def acc():
        c = e.counters()
        for k in sums:
            sums[k] += c[k]
    timer = Timer(torch, stream, dev)
    sampler = ClockSampler(local)
    sampler.start()
    total_ms = timer.run(lambda: batch.step(1), K, acc)
    torch.cuda.synchronize()
    if world_size > 1:
        dist.barrier()
    clocks = sampler.stop()
    c1 = e.counters()
    value, max_s, job_steps = job_rate(torch, dist, world_size, dev, n_bodies * K, total_ms / 1e3)
    max_ms, job_bodies = max_s * 1e3, job_steps / K
    phases = e.phase_times()
    msb = mean_shape_bytes(scene_list)
    bytes_by_phase = step_bytes(msb, sums["pairs"], sums["manifolds"], n_bodies - len(scene_list), K)
    kernel_of = {"solve": "k_color_solve_teams", "narrow": "k_narrow", "integrate": "k_integrate",
                 "pose": "k_collider_pose", "sort": "k_sort_pass", "query": "k_query_stash + k_query_emit"}
    roof = roofline_line(phases, bytes_by_phase, kernel_of, "c4", solve_passes(sums["manifolds"]))
    pose_bytes = e.field_bytes(ag2d.BODY_POSE)
    del batch, e

    # End to end through the C ABI, over the same window: the host checkpoint of the window's start (page-locked)
    # loaded into a resident engine inside the timed region (ag2d_batch_load: the engine's buffers exist, as a
    # server's do between jobs; the upload is timed), then per step one ag2d_batch_step and a read of every body's
    # pose (x, y, rotation) into page-locked host memory. The read of step k is queued after it and lands while
    # step k + 1 runs; the loop waits for it before queuing the next (a consumer one frame behind). The consumer's
    # two page-locked pose buffers exist before the timed region (a viewer allocates them once).
    e2e_steps = K
    pose_ring = [ag2d.host_empty(pose_bytes), ag2d.host_empty(pose_bytes)]
    b2 = ag2d.Batch.restore(ckpt)   # the resident engine (allocation and tuning before the timed region)
    if tuning:
        b2.engine.set_tuning(tuning)
    b2.step(1)                      # its buffers sized by a real step of the window
    allocs0 = ag2d.device_allocs()
    if world_size > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b2.load(ckpt)
    allocs_restore = ag2d.device_allocs() - allocs0
    for k in range(e2e_steps):
        b2.step(1)
        b2.engine.read_wait()
        b2.engine.read_async(ag2d.BODY_POSE, pose_ring[k & 1])
    b2.engine.read_wait()
    torch.cuda.synchronize()
    e2e_s = reduce_max(torch, dist, world_size, dev, time.perf_counter() - t0)
    e2e = {"value": job_bodies * e2e_steps / e2e_s, "unit": METRIC,
           "h2d_bytes_per_step": ckpt.nbytes / e2e_steps, "d2h_bytes_per_step": int(pose_bytes),
           "steps": e2e_steps, "window": window_name(args),
           "timed": "ag2d_batch_load of a page-locked host checkpoint of the window's start into the resident "
                    "engine (in the timed region), then per step ag2d_batch_step + ag2d_world_read_async of every "
                    "body pose into page-locked memory, waited for one step later; wall clock",
           "device_allocs": {"load": allocs_restore,
                             "steps": ag2d.device_allocs() - allocs0 - allocs_restore}}
    del b2, pose_ring

    # The same worlds, one launch sequence per world per step (a Simulation per world): every k-th world.
    per_world_line = None
    if worlds and args.per_world_sample > 0:
        stride = max(1, len(worlds) // args.per_world_sample)
        sample = worlds[::stride]
        for w in sample:
            w.step(args.warmup)
        torch.cuda.synchronize()
        pw_steps = 5
        t0 = time.perf_counter()
        for _ in range(pw_steps):
            for w in sample:
                w.step(1)
        torch.cuda.synchronize()
        pw_s = time.perf_counter() - t0
        pw_bodies = sum(scene_list[k].n for k in range(0, len(worlds), stride))
        per_world = reduce_sum(torch, dist, world_size, dev, pw_bodies * pw_steps / pw_s)
        per_world_line = {"value": per_world, "unit": METRIC,
                          "sample": f"every {stride}-th world ({len(sample)} worlds), steps {args.warmup}.."
                                    f"{args.warmup + pw_steps} from rest, each world its own ag2d_world_step launch "
                                    f"sequence, wall clock (host launch bound; the early steps have fewer contacts "
                                    f"than the batched window, which favours this form)",
                          "batched_over_per_world": value / per_world}
        del sample

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        cpu = cpu_c4(scene_list, start, K)
    return {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world_size, "steps": K, "warmup": W,
        "ms_per_step": max_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32", "data": "synthetic (seeded scene generator, ag2d.scenes.make_c4_worlds)",
        "config": {"workload": WORKLOADS["c4"], "worlds_per_gpu": len(scene_list), "bodies_per_gpu": n_bodies,
                   "window": window_name(args),
                   "parallelism": f"independent worlds x{world_size} GPUs (no step-path collective)",
                   "autotuned": tuning,
                   "steps_before_timing": f"{start - W} settling steps, launch shapes tuned on a copy restored "
                                          f"there, then {W} warm-up steps",
                   "l2": "flushed between timed steps (256 MiB write outside the events)",
                   "mean_pairs_per_step": sums["pairs"] / K, "mean_manifolds_per_step": sums["manifolds"] / K},
        "per_world_launch": per_world_line,
        "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": int(c1["launches"] - c0["launches"]), "clocks": clocks,
        "phase_ms_per_step": {k: round(v[0] / max(K, 1), 4) for k, v in phases.items()},
        "diagnostics": diagnostics(c0, c1, timer.ms, sums["colors"], K),
    }


def run_c2(args, torch, dist, rank, world_size, local, dev):
    import ag2d
    scene = c2_scene(args.bodies)
    w = ag2d.World.from_scene(scene, device=local)
    stream = torch.cuda.ExternalStream(w.stream(), device=dev)
    w.step(args.warmup)
    w.set_profiling(True)
    c0 = w.counters()
    if world_size > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sums = {"pairs": 0, "manifolds": 0, "colors": 0}

    def acc():
        c = w.counters()
        for k in sums:
            sums[k] += c[k]
    timer = Timer(torch, stream, dev)
    sampler = ClockSampler(local)
    sampler.start()
    total_ms = timer.run(lambda: w.step(1), args.steps, acc)
    torch.cuda.synchronize()
    if world_size > 1:
        dist.barrier()
    clocks = sampler.stop()
    c1 = w.counters()
    K = args.steps
    max_ms = reduce_max(torch, dist, world_size, dev, total_ms)
    value = world_size * scene.n * K / (max_ms / 1e3)
    phases = w.phase_times()
    msb = mean_shape_bytes([scene])
    nb, nc = w.counts()
    bytes_by_phase = step_bytes(msb, sums["pairs"], sums["manifolds"], nb - int((scene.mass == 0).sum()), K)
    kernel_of = {"solve": "k_color_solve_cluster", "narrow": "k_narrow", "integrate": "k_integrate",
                 "pose": "k_collider_pose", "sort": "k_sort_pass", "query": "k_query_stash + k_query_emit"}
    roof = roofline_line(phases, bytes_by_phase, kernel_of, "c2", solve_passes(sums["manifolds"]))

    e2e_steps = min(K, 300)
    if world_size > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    w2 = ag2d.World.from_scene(scene, device=local)
    for _ in range(e2e_steps):
        w2.step(1)
        pose = w2.read(ag2d.BODY_POSE)
    torch.cuda.synchronize()
    e2e_s = reduce_max(torch, dist, world_size, dev, time.perf_counter() - t0)
    e2e = {"value": world_size * scene.n * e2e_steps / e2e_s, "unit": METRIC,
           "h2d_bytes_per_step": upload_bytes([scene]) / e2e_steps, "d2h_bytes_per_step": int(pose.nbytes),
           "steps": e2e_steps}
    del pose, w2

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        cpu = cpu_c2(scene, args.cpu_seconds)
    return {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world_size, "steps": K, "warmup": args.warmup,
        "ms_per_step": max_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32", "data": "synthetic (seeded scene generator, ag2d.scenes.make_c2)",
        "config": {"workload": WORKLOADS["c2"], "bodies": scene.n, "colliders": nc,
                   "parallelism": f"replicas x{world_size} (one world per GPU, no step-path collective)",
                   "l2": "flushed between timed steps (256 MiB write outside the events)",
                   "mean_pairs_per_step": sums["pairs"] / K, "mean_manifolds_per_step": sums["manifolds"] / K},
        "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": int(c1["launches"] - c0["launches"]), "clocks": clocks,
        "phase_ms_per_step": {k: round(v[0] / max(K, 1), 4) for k, v in phases.items()},
        "diagnostics": diagnostics(c0, c1, timer.ms, sums["colors"], K),
    }


def run_c3(args, torch, dist, rank, world_size, local, dev):
    import numpy as np
    import ag2d
    from ag2d import roofline
    scene = c3_scene(args.bodies)
    w = ag2d.World.from_scene(scene, device=local)
    stream = torch.cuda.ExternalStream(w.stream(), device=dev)
    w.run_phase(ag2d.PHASE_SPATIAL_FULL)
    for _ in range(args.warmup):
        w.run_phase(ag2d.PHASE_COLLIDE)
    w.set_profiling(True)
    c0 = w.counters()
    if world_size > 1:
        dist.barrier()
    torch.cuda.synchronize()
    timer = Timer(torch, stream, dev)
    sampler = ClockSampler(local)
    sampler.start()
    total_ms = timer.run(lambda: w.run_phase(ag2d.PHASE_COLLIDE), args.steps)
    torch.cuda.synchronize()
    if world_size > 1:
        dist.barrier()
    clocks = sampler.stop()
    c1 = w.counters()
    K = args.steps
    max_ms = reduce_max(torch, dist, world_size, dev, total_ms)
    ms_step = max_ms / K
    value = world_size * scene.n * K / (max_ms / 1e3)
    pairs, mans = c1["pairs"], c1["manifolds"]
    msb = mean_shape_bytes([scene])
    step_b = roofline.broad_narrow_bytes_per_step(scene.n, msb, pairs, mans)
    peak, peak_kind = measured_peaks()
    achieved = step_b / (ms_step / 1e3) / 1e9
    phases = w.phase_times()
    # Exact pair set against the oracle's sweep over the same AABBs.
    aabb = [w.read(f) for f in (ag2d.COL_AABB_MIN_X, ag2d.COL_AABB_MIN_Y, ag2d.COL_AABB_MAX_X, ag2d.COL_AABB_MAX_Y)]
    ours = w.read(ag2d.PAIRS)
    overlap_frac = float(np.unique(ours.reshape(-1)).size) / scene.n if ours.size else 0.0
    try:
        from oracle import oraapi
        ref = oraapi.broad_pairs_from_aabbs(*aabb, np.arange(scene.n, dtype=np.uint32))
        canon = np.sort(ours, axis=1)
        canon = canon[np.lexsort((canon[:, 1], canon[:, 0]))]
        pair_check = {"oracle_pairs": int(ref.shape[0]),
                      "identical_pair_set": bool(ref.shape == canon.shape and np.array_equal(ref, canon))}
    except Exception as exc:  # the oracle library is test infrastructure and may be absent
        pair_check = {"oracle_pairs": None, "identical_pair_set": None, "note": f"oracle unavailable: {exc}"}

    e2e_reps = min(K, 10)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    w2 = ag2d.World.from_scene(scene, device=local)
    w2.run_phase(ag2d.PHASE_SPATIAL_FULL)
    for _ in range(e2e_reps):
        w2.run_phase(ag2d.PHASE_COLLIDE)
        man = w2.read(ag2d.MANIFOLDS)
    torch.cuda.synchronize()
    e2e_s = reduce_max(torch, dist, world_size, dev, time.perf_counter() - t0)
    e2e = {"value": world_size * scene.n * e2e_reps / e2e_s, "unit": METRIC,
           "h2d_bytes_per_step": upload_bytes([scene]) / e2e_reps, "d2h_bytes_per_step": int(man.nbytes),
           "steps": e2e_reps}
    del w2, man

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        r = cpu_c3(scene, 3)
        if r:
            cpu = {"value": scene.n / r["seconds"], "unit": METRIC, "cores": r["threads"], "kind": "reference",
                   "sample": f"reference engine collision detection (spatial data, broad, narrow; "
                             f"agref_timed_collide) on the same {scene.n}-body world, median of 3 passes, "
                             f"{r['seconds'] * 1e3:.1f} ms; its pair count {r['pairs']}",
                   "gbs_equivalent": step_b / r["seconds"] / 1e9}
    return {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world_size, "steps": K, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
        "data": "synthetic (seeded scene generator, ag2d.scenes.make_c3)",
        "config": {"workload": WORKLOADS["c3"], "bodies": scene.n, "pairs": pairs, "manifolds": mans,
                   "fraction_of_bodies_with_overlap": overlap_frac, "pair_check": pair_check,
                   "l2": "flushed between timed passes (256 MiB write outside the events)"},
        "broadphase_gbs": achieved,
        "roofline": {"bound": "hbm", "kernel": "collision detection pass (pose, bounds, Morton, sort, LBVH, query, "
                                                "narrow, compaction)", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)", "traffic": None,
                     "algorithmic_bytes_per_launch": step_b},
        "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": int(c1["launches"] - c0["launches"]), "clocks": clocks,
        "phase_ms_per_step": {k: round(v[0] / max(K, 1), 4) for k, v in phases.items()},
    }


def run_c5(args, torch, dist, rank, world_size, local, dev):
    """Serving: arrivals replayed on a wall clock by a submitter thread; the server admits, steps and retires the
    requests on its own host thread. Worlds are built on the host before the run (request construction is the
    client's work); each submit copies the world's arrays into the request. Every rank serves its own stream."""
    import ag2d
    import numpy as np
    n_req = args.requests
    scene_list = c5_requests(n_req, rank_seed(rank, 1_000_003))
    warm_list = c5_requests(32, rank_seed(rank, 1_000_003) + 777)
    arrivals = poisson_arrivals(n_req, args.rate, rank)
    settings = dict(dt=scene_list[0].dt, velocity_iterations=8, position_iterations=3,
                    gravity=scene_list[0].gravity, ccd=True, device=local)

    def build(lst):
        out = []
        for sc in lst:
            w = ag2d.World(**settings)
            w.add_scene(sc)
            out.append(w)
        return out
    worlds, warm = build(scene_list), build(warm_list)
    server = ag2d.Server(memory_budget_bytes=int(args.budget_gb * (1 << 30)), steps_per_round=args.round_steps,
                         reserve_bodies=args.reserve_bodies, **settings)
    # Warm-up: a burst of requests through the same server (allocations, first launches).
    for w in warm:
        server.submit(w, args.steps)
    server.wait_all(600_000)
    s0 = server.stats()
    if world_size > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    ids = [0] * n_req
    lag = [0.0]

    def submitter():
        t_start = time.perf_counter()
        for k in range(n_req):
            delay = arrivals[k] - (time.perf_counter() - t_start)
            if delay > 0:
                time.sleep(delay)
            else:
                lag[0] = max(lag[0], -delay)
            ids[k] = server.submit(worlds[k], args.steps)
    t0 = time.perf_counter()
    th = threading.Thread(target=submitter)
    th.start()
    th.join()
    server.wait_all(1_800_000)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    clocks = sampler.stop()
    s1 = server.stats()
    lat = np.array([server.poll(i)[1] for i in ids])
    bodies = int(sum(sc.n for sc in scene_list))
    body_steps = bodies * args.steps
    value, max_wall, job = job_rate(torch, dist, world_size, dev, body_steps, wall)
    p50, p99 = float(np.percentile(lat, 50)), float(np.percentile(lat, 99))
    served_rate = n_req / wall
    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        from oracle import refapi
        if refapi.available():
            sample = scene_list[:512]
            threads = host_threads()
            v = cpu_worlds_rate(sample, args.cpu_seconds, threads, max_steps=args.steps, ccd=True)
            cpu = {"value": v, "unit": METRIC, "cores": threads, "kind": "reference",
                   "sample": f"reference engine (oracle/_ref), the first {len(sample)} requests, one single-threaded "
                             f"Simulation each with CCD, {threads} at a time, {args.steps} steps each, "
                             f"{args.cpu_seconds:.0f} s of serving"}
    req_bytes = upload_bytes(scene_list) / n_req
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world_size, "steps": args.steps,
        "warmup": len(warm), "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32", "data": "synthetic (seeded request generator, ag2d.scenes.make_c5_requests)",
        "config": {"workload": WORKLOADS["c5"], "requests_per_gpu": n_req, "bodies_per_gpu": bodies,
                   "rate_per_s": args.rate, "budget_gb": args.budget_gb, "round_steps": args.round_steps,
                   "reserve_bodies": args.reserve_bodies,
                   "parallelism": f"one server per GPU x{world_size} (no collective)",
                   "timing": "wall clock from the first arrival to the last completion (arrivals follow a wall "
                             "clock); warm-up: a burst of 32 requests through the same server",
                   "l2": "inputs larger than L2 (the resident batch)"},
        "latency_ms": {"p50": p50, "p99": p99, "max": float(lat.max()), "mean": float(lat.mean())},
        "serving": {"offered_body_steps_per_s": args.rate * bodies * args.steps / n_req,
                    "served_requests_per_s": served_rate, "rounds": s1["rounds"] - s0["rounds"],
                    "peak_resident": s1["peak_resident"], "server_busy_ms": s1["busy_ms"] - s0["busy_ms"],
                    "server_step_ms": s1["step_ms"] - s0["step_ms"], "server_repack_ms": s1["repack_ms"] - s0["repack_ms"],
                    "submit_lag_ms": 1e3 * lag[0]},
        "roofline": None,
        "roofline_note": "per-kernel roofline is reported on the c4 and c3 lines; this line measures serving",
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_request": req_bytes,
                "d2h_bytes_per_request": 36.0 * bodies / n_req,
                "note": "the serving run is end to end: host worlds in, host results out"},
        "clocks": clocks,
    }
    server.close()
    return line


def extra_args(args, workload):
    """Arguments of a sub-run of the default line: the workload's own defaults, shortened where they are long."""
    a = argparse.Namespace(**vars(args))
    a.workload = workload
    if workload == "c3":
        a.steps, a.bodies, a.warmup = 20, 1_000_000, max(3, args.warmup)
    else:
        a.steps, a.requests, a.cpu_seconds = DEFAULT_STEPS["c5"], args.extra_requests, min(args.cpu_seconds, 10.0)
    return a


def pick(d, keys):
    return {k: d[k] for k in keys if k in d}


def run_ours(args):
    import torch
    import torch.distributed as dist

    rank, world_size, local = dist_env()
    if world_size > 1:
        import datetime
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device(f"cuda:{local}")
    fn = {"c4": run_c4, "c2": run_c2, "c3": run_c3, "c5": run_c5}[args.workload]
    line = fn(args, torch, dist, rank, world_size, local, dev)
    if args.workload == "c4" and not args.no_extras:
        # The rest of the headline metric: broad+narrow GB/s of the 1M-body pass and the serving latency.
        import gc
        gc.collect()
        torch.cuda.synchronize()
        c3 = run_c3(extra_args(args, "c3"), torch, dist, rank, world_size, local, dev)
        line["c3"] = pick(c3, ("value", "unit", "ms_per_step", "broadphase_gbs", "roofline", "cpu_baseline",
                               "e2e", "gpu_launches", "clocks", "phase_ms_per_step"))
        line["c3"]["config"] = c3["config"]
        gc.collect()
        c5 = run_c5(extra_args(args, "c5"), torch, dist, rank, world_size, local, dev)
        line["c5"] = pick(c5, ("value", "unit", "latency_ms", "serving", "cpu_baseline", "clocks", "config"))
        line["broadphase_gbs"] = c3["broadphase_gbs"]
        line["broadphase_roofline_frac"] = c3["roofline"]["frac"]
        line["serving_p50_ms"] = c5["latency_ms"]["p50"]
        line["serving_p99_ms"] = c5["latency_ms"]["p99"]
    if rank == 0:
        print(json.dumps(line))
    if world_size > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
