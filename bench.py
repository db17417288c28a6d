#!/usr/bin/env python
"""Benchmark driver: one JSON line per run on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Workloads (synthetic inputs with the reference scenes' shapes; the reference
publishes no numbers, so vs_baseline is null):

* ``dito``     - DiTO-14 fit of 100,000,000 points on an ellipsoid surface
                 (semi-axes 4, 1, 0.25; rotated, noised, offset).  A step is
                 one fit: two streaming passes.  Metric Mpoints/s.

Multi-GPU: every rank fits its own point set (independent units, no
collective); ``value`` is the points of all ranks over the slowest rank's
device time ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import ctypes
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["dito"], default="dito")
    ap.add_argument("--points", type=int, default=100_000_000)
    ap.add_argument("--profile", action="store_true",
                    help="only warm-up + timed fits, no clock soak, e2e or CPU legs (for ncu captures)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.file = None

    def start(self):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu)], stdout=self.file, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r.strip() for r in self.file.read().splitlines() if r.strip()]
        self.file.close()
        os.unlink(self.file.name)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            c = [x.strip() for x in r.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1]))
                smax.append(float(c[2]))
            except ValueError:
                continue
            for name, v in zip(names, c[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False

    def init(self, backend="nccl"):
        import torch
        if self.world > 1:
            import torch.distributed as dist
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.pg = True
        elif backend == "nccl":
            torch.cuda.set_device(0)

    def barrier(self):
        if self.pg:
            import torch.distributed as dist
            dist.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            import torch.distributed as dist
            dist.destroy_process_group()


# ---------------------------------------------------------------------------
def cpu_reference_dito(points_np, repeats: int):
    """The reference's own DiTO_14 (oracle/_ref) on host cores: Mpoints/s."""
    import oracle
    oracle.ref_dito14(points_np[:1000])
    t0 = time.perf_counter()
    for _ in range(repeats):
        oracle.ref_dito14(points_np)
    dt = time.perf_counter() - t0
    return points_np.shape[0] * repeats / dt / 1e6, dt


def bench_dito_ours(a, dist: Dist):
    import torch
    from obvh_b200 import DitoFitter, points_obb, workloads

    n = a.points
    dev = torch.device("cuda", torch.cuda.current_device())
    # Two independent point sets, alternated between steps: a step never finds
    # the previous step's data in L2 (each set is 1.2 GB, the L2 126 MB).
    sets = [workloads.ellipsoid_points_torch(n, seed=1234 + 2 * dist.rank + j, device=dev) for j in range(2)]
    pts = sets[0]
    fitter = DitoFitter(dev)
    out = torch.empty(15, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    sampler = ClockSampler(dev.index if dist.world == 1 else dist.local)
    if not a.profile:
        sampler.start()
        # settle clocks: ~1 s of back-to-back fits before the warm-up
        t_end = time.time() + 1.0
        while time.time() < t_end:
            for j in range(20):
                fitter.fit(sets[j & 1], out)
            torch.cuda.synchronize()
    for j in range(a.warmup):
        fitter.fit(sets[j & 1], out)
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()

    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
            torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for j, (e0, e1, e2) in enumerate(evs):
        p = sets[(j + a.warmup) & 1]
        e0.record(stream)
        fitter.fit_pass(p, out, 1)
        e1.record(stream)
        fitter.fit_pass(p, out, 2)
        e2.record(stream)
    stop.record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    clocks = sampler.stop() if not a.profile else None

    total_ms = dist.max(start.elapsed_time(stop))
    p1 = [e0.elapsed_time(e1) for e0, e1, _ in evs]
    p2 = [e1.elapsed_time(e2) for _, e1, e2 in evs]
    ms_step = total_ms / a.steps
    value = dist.world * n * a.steps / (total_ms / 1e3) / 1e6

    path, _, err = fitter.report()
    if err:
        raise RuntimeError(f"device error word {err}")
    if a.profile:
        return {"profile": "dito", "points": n, "pass1_ms": statistics.mean(p1), "pass2_ms": statistics.mean(p2),
                "path": path}

    peak, peak_kind = peaks()
    t1, t2 = statistics.mean(p1), statistics.mean(p2)
    dom_name, dom_ms = ("dito_extremal_pass", t1) if t1 >= t2 else ("dito_extent_pass", t2)
    algo_bytes = 12.0 * n  # one pass reads every point once
    achieved = algo_bytes / (dom_ms / 1e3) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "dito_traffic.json")
    if os.path.exists(prof):
        with open(prof) as f:
            tj = json.load(f)
        if dom_name in tj:
            traffic = tj[dom_name]["bytes_per_point"] * n

    # End to end through the reference-facing call: host (pinned) points in,
    # box out; the H2D copy of the points and the read-back are inside.
    host = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
    host.copy_(pts)
    host_np = host.numpy()
    points_obb(host_np)  # warm
    e2e_steps = max(3, min(a.steps, 10))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        points_obb(host_np)
    e2e_s = time.perf_counter() - t0
    e2e_local = n * e2e_steps / e2e_s / 1e6
    e2e_min = -dist.max(-e2e_local)

    line = {
        "metric": "DiTO-14 fit throughput (Mpoints/s)",
        "value": round(value, 3),
        "unit": "Mpoints/s",
        "n_gpus": dist.world,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": round(ms_step, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic: ellipsoid surface points (4,1,0.25), Haar rotation, N(0,0.01^2) noise, U[-10,10]^3 offset",
        "config": {"workload": "dito_plain_fit", "points_per_gpu": n, "point_bytes": 12,
                   "l2": "two 1.2 GB point sets alternated between steps (> 126 MB L2), no flush", "parallelism": f"replicas{dist.world}",
                   "path": path},
        "kernels_ms": {"dito_extremal_pass": round(t1, 5), "dito_extent_pass": round(t2, 5)},
        "gpu_launches": 2 * a.steps,
        "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": round(achieved, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                     "peak_source": peak_kind, "algorithmic_bytes_per_launch": algo_bytes},
        "e2e": {"value": round(dist.world * e2e_min, 3), "unit": "Mpoints/s", "h2d_bytes_per_step": 12 * n,
                "d2h_bytes_per_step": 316, "api": "obvh_points_obb (kr_cuda_points_obb with errors), pinned host"},
        "clocks": clocks,
    }
    if dist.rank == 0 and dist.world == 1:
        sample = host_np[: min(n, 100_000_000)]
        v, dt = cpu_reference_dito(sample, repeats=3)
        line["cpu_baseline"] = {"value": round(v, 3), "unit": "Mpoints/s", "cores": 1, "kind": "reference",
                                "sample": f"3 fits of the first {sample.shape[0]} points ({dt:.1f} s)"}
    return line


def bench_dito_reference(a, dist: Dist):
    """The reference's own CPU DiTO_14 (single-threaded, as shipped) on this host."""
    import numpy as np
    import oracle
    from obvh_b200 import workloads
    n = a.points
    try:
        import torch
        pts = workloads.ellipsoid_points_torch(n, seed=1234, device="cuda" if torch.cuda.is_available() else "cpu")
        host = pts.cpu().numpy()
    except Exception:
        host = workloads.ellipsoid_points(n, seed=1234)
    host = np.ascontiguousarray(host, dtype=np.float32)
    for _ in range(a.warmup):
        oracle.ref_dito14(host)
    times = []
    for _ in range(a.steps):
        t0 = time.perf_counter()
        oracle.ref_dito14(host)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = n * a.steps / total / 1e6
    return {
        "metric": "DiTO-14 fit throughput (Mpoints/s)", "impl": "reference", "value": round(value, 3),
        "unit": "Mpoints/s", "n_gpus": dist.world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": round(1e3 * total / a.steps, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (same generator as the ours arm)",
        "config": {"workload": "dito_plain_fit", "points_per_gpu": n},
        "cpu_baseline": {"value": round(value, 3), "unit": "Mpoints/s", "cores": 1, "kind": "reference",
                         "sample": f"full {n}-point fit per step; DiTO_14<float> is single-threaded"},
        "e2e": {"value": round(value, 3), "unit": "Mpoints/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    a = parse_args()
    dist = Dist()
    if a.impl == "reference":
        if dist.world > 1 and dist.rank != 0:
            return
        import oracle
        if not oracle.ref_available():
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_dito.so was not built"}))
            return
        print(json.dumps(bench_dito_reference(a, dist)), flush=True)
        return
    dist.init("nccl")
    try:
        line = bench_dito_ours(a, dist)
        if dist.rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
