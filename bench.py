#!/usr/bin/env python
"""Throughput of the collision/contact pipeline on B200: body-steps/s of the single large world (100,000 mixed
bodies, U container, dt 1/60, 8 velocity + 3 position iterations), stepped from the drop.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--bodies n]

One process per GPU (torchrun for N > 1): a single world does not shard without a halo exchange, so every rank
steps its own replica of the world (replicas only, no collective on the step path) and the whole-job value is
N x bodies x K / (the slowest rank's device time). Rank 0 prints one JSON line.

Timing: W untimed warm-up steps, then K steps, each bracketed by CUDA events on the world's stream, with a 256 MiB
write between steps (L2 flushed; the timed region excludes it); barrier + synchronize around the timed region; the
max over ranks. SM clocks are sampled with nvidia-smi during the timed region. The end-to-end number goes through
the C ABI with host buffers: the scene uploaded from host memory, then per step one ag2d_world_step and one
readback of every body's pose into host memory.

--impl reference times the reference engine itself (oracle/_ref/libagony_ref.so, its own C++ on the host cores,
all threads) on the same workload and prints the same line with "impl": "reference".
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "physicssimulation-agony_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "body-steps/s"
WORKLOAD = "c2: single large world, 100k mixed bodies (60% boxes, 25% circles, 15% 3-8-gons) in a static U, " \
           "dt 1/60, 8 velocity + 3 position iterations, stepped from the drop"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--bodies", type=int, default=100_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def make_scene(n):
    from ag2d import scenes
    cols = 500 if n >= 100_000 else max(10, int(round((n / 200.0) ** 0.5 * 10)))
    return scenes.make_c2(n, 0, columns=cols)


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


def mean_shape_bytes(scene):
    from ag2d import roofline, scenes
    total = 0.0
    for k in range(scene.n):
        kind = int(scene.kind[k])
        total += roofline.polygon_bytes(int(scene.poly_count[k])) if kind == scenes.POLYGON else \
            roofline.SHAPE_BYTES[kind]
    return total / max(scene.n, 1)


def cpu_baseline(scene, seconds):
    """The reference engine (its own C++, all host threads) on the first steps of the same workload."""
    from oracle import refapi
    if not refapi.available():
        return None
    threads = max(0, (os.cpu_count() or 1) - 1)
    sim = refapi.RefSim(scene, threads=threads)
    steps, elapsed = 0, 0.0
    while elapsed < seconds and steps < 100000:
        elapsed += sim.timed_update(1)
        steps += 1
    sim.close()
    return {"value": scene.n * steps / elapsed, "unit": METRIC, "cores": threads + 1, "kind": "reference",
            "sample": f"reference engine (oracle/_ref, -O2 -mavx2 -mfma) on the first {steps} steps of the same "
                      f"{scene.n}-body world from the drop, {threads + 1} threads, {elapsed:.1f} s wall"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import refapi
    if not refapi.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libagony_ref.so was not built"}))
        return
    scene = make_scene(args.bodies)
    threads = max(0, (os.cpu_count() or 1) - 1)
    sim = refapi.RefSim(scene, threads=threads)
    sim.update(args.warmup)
    budget = 150.0
    steps, elapsed = 0, 0.0
    while steps < args.steps and elapsed < budget:
        elapsed += sim.timed_update(1)
        steps += 1
    sim.close()
    value = scene.n * steps / elapsed
    sample = f"steps {args.warmup}..{args.warmup + steps} of the {scene.n}-body world ({threads + 1} threads)"
    if steps < args.steps:
        sample += f"; stopped after {budget:.0f} s of {args.steps} requested steps"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 0, "steps": steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / max(steps, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "bodies": scene.n},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads + 1, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_ours(args):
    import torch
    import torch.distributed as dist

    import ag2d
    from ag2d import roofline

    rank, world_size, local = dist_env()
    if world_size > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device(f"cuda:{local}")

    scene = make_scene(args.bodies)
    w = ag2d.World.from_scene(scene, device=local)
    stream = torch.cuda.ExternalStream(w.stream(), device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)   # 256 MiB > 126 MB L2

    w.step(args.warmup)
    w.set_profiling(True)
    c0 = w.counters()
    if world_size > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    per_step = []
    pairs_sum = manifolds_sum = colors_sum = 0
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        w.step(1)
        e1.record(stream)
        e1.synchronize()
        per_step.append(e0.elapsed_time(e1))
        c = w.counters()
        pairs_sum += c["pairs"]
        manifolds_sum += c["manifolds"]
        colors_sum += c["colors"]
    torch.cuda.synchronize()
    if world_size > 1:
        dist.barrier()
    clocks = sampler.stop()
    c1 = w.counters()
    total_ms = float(sum(per_step))
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if world_size > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    value = world_size * scene.n * args.steps / (max_ms / 1e3)
    phases = w.phase_times()

    # Dominant single-kernel phase and its roofline (algorithmic bytes / measured kernel time).
    K = args.steps
    msb = mean_shape_bytes(scene)
    nb, nc = w.counts()
    dyn_bodies = nb - int((scene.mass == 0).sum())
    bytes_by_phase = {
        "solve": roofline.solve_bytes(manifolds_sum, 8, 3),
        "narrow": roofline.narrow_bytes(pairs_sum, msb, manifolds_sum),
        "integrate": roofline.integrate_bytes(dyn_bodies * K),
        "pose": roofline.pose_bytes(dyn_bodies * K, msb),
        "sort": roofline.sort_bytes(dyn_bodies * K),
        "query": roofline.query_bytes(dyn_bodies * K, pairs_sum),
    }
    kernel_of = {"solve": "k_solve", "narrow": "k_narrow", "integrate": "k_integrate", "pose": "k_collider_pose",
                 "sort": "k_sort_pass", "query": "k_query_count + k_query_write"}
    dominant = max(bytes_by_phase, key=lambda p: phases[p][0])
    peak, peak_kind = measured_peaks()
    dom_ms, dom_calls = phases[dominant]
    achieved = bytes_by_phase[dominant] / max(dom_ms / 1e3, 1e-12) / 1e9
    traffic = None
    prof_path = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if os.path.exists(prof_path):
        try:
            traffic = json.load(open(prof_path)).get(kernel_of[dominant])
        except (OSError, ValueError):
            traffic = None

    # End to end through the C ABI: scene upload from host memory, then per step a step + a pose readback.
    w2 = ag2d.World.from_scene(scene, device=local)
    e2e_steps = min(K, 300)
    h2d = scene.n * (4 * 4 + 4 * 4 + 8 + 12) + int(scene.poly_count.sum()) * 16
    if world_size > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    w2.step(1)          # first step uploads the host scene
    pose = w2.read(ag2d.BODY_POSE)
    for _ in range(e2e_steps - 1):
        w2.step(1)
        pose = w2.read(ag2d.BODY_POSE)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if world_size > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world_size * scene.n * e2e_steps / float(te.item())
    del pose, w2

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(scene, args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world_size, "steps": K,
            "warmup": args.warmup, "ms_per_step": max_ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32", "data": "synthetic (seeded scene generator, ag2d.scenes.make_c2)",
            "config": {"workload": WORKLOAD, "bodies": scene.n, "colliders": nc,
                       "parallelism": f"replicas x{world_size} (one world per GPU, no step-path collective)",
                       "l2": "flushed between timed steps (256 MiB write outside the events)",
                       "mean_pairs_per_step": pairs_sum / K, "mean_manifolds_per_step": manifolds_sum / K},
            "roofline": {"bound": "hbm", "kernel": kernel_of[dominant], "phase": dominant, "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": traffic, "launch_ms": dom_ms / max(dom_calls, 1)},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d / e2e_steps,
                    "d2h_bytes_per_step": scene.n * 16, "steps": e2e_steps},
            "gpu_launches": int(c1["launches"] - c0["launches"]),
            "clocks": clocks,
            "phase_ms_per_step": {k: round(v[0] / max(K, 1), 4) for k, v in phases.items()},
            "diagnostics": {"mean_colors": colors_sum / K,
                            "list_rebuilds": c1["list_rebuilds"] - c0["list_rebuilds"],
                            "retries": c1["retries"] - c0["retries"], "regrows": c1["regrows"] - c0["regrows"],
                            "host_ms_per_step": (c1["host_ms"] - c0["host_ms"]) / K,
                            "sync_wait_ms_per_step": (c1["sync_ms"] - c0["sync_ms"]) / K,
                            "max_step_ms": max(per_step), "median_step_ms": statistics.median(per_step)},
        }
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
