#!/usr/bin/env python
"""Benchmark driver: one JSON line per run on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Workloads (seeded synthetic inputs with the reference scenes' shapes; the
reference publishes no numbers, so vs_baseline is null):

* ``lbvh_obb_tree`` (default) - LBVH (30-bit Morton, Karras, 1 primitive per
  leaf) over 2,000,000 thin random triangles (centroids uniform in [0,1]^3,
  vertices at log-uniform radius 0.002..0.02), then the AABB->OBB-tree
  transform, then the node collapse.  A step is one such build.  Metric
  Mnodes/s = (2N-1) nodes per step.
* ``atrbvh_obb_tree`` - ATRBVH (63-bit Morton LBVH, then agglomerative
  treelet optimisation, treelet size 7, 2 iterations) over the 917,504-triangle
  (2,3) torus-knot tube, then the OBB-tree transform and the collapse.  A step
  is one such build.  Metric Mnodes/s.
* ``dito`` - DiTO-14 fit of 100,000,000 points on an ellipsoid surface
  (semi-axes 4, 1, 0.25; rotated, noised, offset).  A step is one fit (two
  streaming passes).  Metric Mpoints/s.
* ``dito_batch`` - DiTO-14 fits of 4,096 anisotropic Gaussian clouds of
  log-uniform sizes 64..262,144 (about 129M points in one CSR buffer) in one
  persistent work-stealing launch replayed from a CUDA graph, knobs picked by
  the autotuner first.  A step is the whole batch.  Metric Mpoints/s; the line
  also carries the plain per-call throughput (one obvh_dito_fit_async per set)
  on the same device-resident buffer.

Multi-GPU: every rank builds/fits its own input (independent units, no
collective); ``value`` = units of all ranks / the slowest rank's device time
("scaling": "weak").
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
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["lbvh_obb_tree", "atrbvh_obb_tree", "dito", "dito_batch", "serve",
                                           "obvh_pack", "obvh_trace", "obvh_trace_compressed", "mesh_batch"],
                    default="lbvh_obb_tree")
    ap.add_argument("--treelet", type=int, default=7, help="atrbvh_obb_tree: treelet size")
    ap.add_argument("--requests", type=int, default=300, help="serve: requests in the stream")
    ap.add_argument("--sets", type=int, default=4096, help="dito_batch: point sets per batch")
    ap.add_argument("--meshes", type=int, default=2048, help="mesh_batch: meshes per batch")
    ap.add_argument("--no-autotune", action="store_true", help="dito_batch: default knobs")
    ap.add_argument("--points", type=int, default=100_000_000, help="dito: points per fit")
    ap.add_argument("--tris", type=int, default=2_000_000, help="lbvh_obb_tree: triangles per build")
    ap.add_argument("--rays", type=int, default=4_000_000, help="obvh_trace: rays per pass")
    ap.add_argument("--profile", action="store_true",
                    help="only warm-up + timed steps, no clock soak, e2e or CPU legs (for ncu captures)")
    ap.add_argument("--no-extras", action="store_true",
                    help="lbvh_obb_tree at 1 GPU: leave out the DiTO-100M, batch and serve sub-objects")
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

    def __init__(self, gpu_index: int, enabled: bool = True):
        self.gpu = gpu_index
        self.enabled = enabled
        self.proc = None
        self.file = None

    def start(self):
        if not self.enabled:
            return
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu)], stdout=self.file, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if not self.enabled or self.file is None:
            return None
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


class Dist:
    """One process per GPU (replicas): a barrier and a max over ranks, nothing
    on the data path.  NCCL on GPUs; gloo when OBVH_DIST_BACKEND=gloo (the CPU
    tests of this plumbing)."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = os.environ.get("OBVH_DIST_BACKEND", "nccl")
        self.pg = False

    def init(self):
        import torch
        if self.backend != "gloo":
            torch.cuda.set_device(self.local if self.world > 1 else 0)
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(self.backend, timeout=datetime.timedelta(seconds=120))
            self.pg = True

    def barrier(self):
        if self.pg:
            import torch.distributed as dist
            dist.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device="cpu" if self.backend == "gloo" else "cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            import torch.distributed as dist
            dist.destroy_process_group()


def profile_summary():
    from obvh_b200 import _native
    buf = ctypes.create_string_buffer(1 << 16)
    _native.check(_native.lib().obvh_profile_summary(buf, len(buf)))
    return json.loads(buf.value.decode())


def profile_enable(on: bool):
    from obvh_b200 import _native
    _native.check(_native.lib().obvh_profile_enable(1 if on else 0))


def timed_steps(a, dist, step_fn, sampler, stream, profile=True):
    """Warm-up, then exactly a.steps steps between barriers; returns the max-over-ranks
    device time (ms), the per-kernel profile of the timed region (an event pair
    around every launch; empty with profile=False) and the clocks."""
    import torch
    if not a.profile:
        sampler.start()
        t_end = time.time() + 1.0  # settle clocks
        j = 0
        while time.time() < t_end:
            step_fn(j)
            j += 1
            torch.cuda.synchronize()
    for j in range(a.warmup):
        step_fn(j)
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    profile_enable(profile)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for j in range(a.steps):
        step_fn(a.warmup + j)
    stop.record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    clocks = sampler.stop() if not a.profile else None
    prof = profile_summary()
    profile_enable(False)
    return dist.max(start.elapsed_time(stop)), prof, clocks


def kernel_table(prof, steps, bytes_per_launch, peak):
    """Per kernel: launches and device time per step, and, where its
    algorithmic bytes are known, the HBM throughput they imply over its
    launch time and that as a fraction of the measured peak."""
    out = {}
    for k, (launches, total_ms) in prof.items():
        e = {"launches": launches, "ms_per_step": round(total_ms / steps, 5)}
        algo = bytes_per_launch.get(k)
        if algo and launches and total_ms > 0:
            gbs = algo / (total_ms / launches / 1e3) / 1e9
            e["algorithmic_gbs"] = round(gbs, 1)
            e["frac"] = round(gbs / peak, 4)
        out[k] = e
    return out


def roofline(prof, bytes_per_launch, peak, peak_kind, traffic_file=None):
    """The roofline object of the kernel with the largest device time."""
    name, (launches, total_ms) = max(prof.items(), key=lambda kv: kv[1][1])
    per_launch_ms = total_ms / max(launches, 1)
    algo = bytes_per_launch.get(name)
    achieved = algo / (per_launch_ms / 1e3) / 1e9 if algo else None
    traffic = None
    if traffic_file and os.path.exists(traffic_file):
        with open(traffic_file) as f:
            traffic = json.load(f).get(name)
    return {"bound": "hbm", "kernel": name, "achieved": round(achieved, 1) if achieved else None, "peak": peak,
            "unit": "GB/s", "frac": round(achieved / peak, 4) if achieved else None, "traffic": traffic,
            "peak_source": peak_kind, "algorithmic_bytes_per_launch": algo,
            "launches": launches, "ms_per_launch": round(per_launch_ms, 5)}


# ---------------------------------------------------------------------------
def tree_bytes_per_launch(n):
    """Algorithmic (compulsory HBM) bytes per launch of each kernel of the
    LBVH -> OBB-tree -> collapse step for n triangles (nn = 2n-1 nodes):
    every input read once and every output written once."""
    ni = n - 1
    nn = 2 * n - 1
    return {
        "tri_bounds_kernel": 52 * n + 24 * n,          # face + 3 vertices in, triangle box out
        "morton_count_kernel": 24 * n + 8 * n,         # box in, key + index out (digits counted on the way)
        "radix_digit_counts": 4 * n,                   # keys in (every pass's digits at once)
        "radix_onesweep": 16 * n,                      # key + value in and out (u32 keys)
        "leaves_kernel": 4 * n + 24 * n + 36 * n,      # order, box in; leaf node out
        "karras_kernel": 4 * n + 36 * ni + 16 * ni,    # codes in; internal nodes, parents, first leaves, spans out
        "aabb_up_kernel": 36 * nn + 8 * nn + 32 * ni,  # nodes in; counts, costs, bounds out
        # faces + vertices in, leaf boxes + transforms out, summaries out and read once
        "summary_up_kernel": 52 * n + 124 * n + 112 * ni * 2 + 4 * ni,
        "dfs_rank_kernel": 52 * n + 36 * n + 4 * ni,   # faces + vertices in; ordered triangles + firsts out
        "candidate_kernel": 112 * ni + 168 * ni + 96 * ni + 8 * ni,  # summary + 14 vertices in; frame out
        "extents_small_kernel": 96 * ni + 124 * ni,    # frame in; box + transform out
        "extents_units_kernel": 36 * n,                # ordered triangles in
        # tiles: ordered triangles, frames, first leaves and counts in; boxes + transforms (or extent keys) out
        "extents_tile_kernel": 36 * n + 104 * ni + 124 * ni,
        "mark_up_kernel": 36 * nn + 16 * nn + 36 * n,
        # fused build: order, face, vertices in; leaf node (x2), ordered triangle, leaf box + transform out
        "leaves_fused_kernel": 4 * n + 52 * n + 72 * n + 36 * n + 124 * n,
        # fused leaf-to-root pass over the CTA-local nodes: triangles in (the leaf bounds are recomputed from
        # them), leaf costs + counts out; children, first leaf, count in; bounds, collapsed node, cost, summary
        # out; collapse marks
        "fused_up_local_kernel": 36 * n + 8 * n + 16 * ni + 24 * ni + 36 * ni + 4 * ni + 112 * ni + nn,
        # ATRBVH: triangle in, 63-bit key + index out; sorted keys in, working nodes out;
        # leaf triangles + nodes in/out bottom-up; one pass over the working tree per iteration
        "morton63_kernel": 52 * n + 12 * n,
        "karras63_kernel": 12 * n + 48 * nn,
        "boxes_up_kernel": 52 * n + 48 * nn * 2,
        "treelet_kernel": 48 * nn * 2 + 8 * nn * 2,
        "emit_kernel": 48 * nn + 36 * nn + 4 * nn,
        "roots_kernel": 14 * nn,
        # ATRBVH commit walk: leaf records, faces and vertices in; bounds, collapsed records, counts, costs,
        # summaries, leaf boxes + transforms and marks out
        "walk_kernel": 36 * n + 52 * n + 24 * ni + 36 * nn + 8 * nn + 112 * ni + 124 * n + nn,
        "gather_kernel": 8 * nn,
        "gather_ranked_kernel": 8 * nn,
        "scan_tile_sums": 4 * nn,
        "scan_tiles": 8 * nn,
    }


def bench_tree_ours(a, dist, atrbvh=False):
    import numpy as np
    import torch
    from obvh_b200 import _native, bvh, workloads

    dev = torch.device("cuda", torch.cuda.current_device())
    lib = _native.lib()
    if atrbvh:
        # two knots alternated between steps (different surface noise)
        host_meshes = [workloads.torus_knot_mesh(seed=2 + 2 * dist.rank + j) for j in range(2)]
        ws_bytes, ws_init, status_fn = lib.obvh_atrbvh_workspace_bytes, lib.obvh_atrbvh_workspace_init, \
            lib.obvh_atrbvh_status
    else:
        # two meshes alternated between steps (2 x 104 MB > 126 MB L2)
        host_meshes = [workloads.triangle_soup(a.tris, seed=1 + 2 * dist.rank + j) for j in range(2)]
        ws_bytes, ws_init, status_fn = lib.obvh_build_workspace_bytes, lib.obvh_build_workspace_init, \
            lib.obvh_build_status
    n = host_meshes[0][1].shape[0]
    nn = 2 * n - 1
    meshes = [bvh.Mesh(v, f, device=dev) for v, f in host_meshes]
    ws = torch.empty(int(ws_bytes(n)), dtype=torch.uint8, device=dev)
    _native.check(ws_init(ctypes.c_void_p(ws.data_ptr()), n, None))
    u8, i32, f32 = torch.uint8, torch.int32, torch.float32
    out = {"nodes": torch.empty(nn * 36, dtype=u8, device=dev), "parents": torch.empty(nn, dtype=i32, device=dev),
           "counts": torch.empty(nn, dtype=i32, device=dev), "costs": torch.empty(nn, dtype=f32, device=dev),
           "bounds": torch.empty(12, dtype=f32, device=dev), "obbs": torch.empty(nn * 15, dtype=f32, device=dev),
           "xfs": torch.empty(nn * 16, dtype=f32, device=dev), "collapsed": torch.empty(nn * 36, dtype=u8, device=dev),
           "prims": torch.empty(n, dtype=i32, device=dev)}
    P = {k: ctypes.c_void_p(t.data_ptr()) for k, t in out.items()}
    W = ctypes.c_void_p(ws.data_ptr())
    stream = torch.cuda.current_stream(dev)
    S = ctypes.c_void_p(stream.cuda_stream)

    flags = bvh.BUILD_OBBS | bvh.BUILD_COLLAPSE

    def step(j, mesh=None):
        m = mesh or meshes[j & 1]
        V, F = ctypes.c_void_p(m.verts.data_ptr()), ctypes.c_void_p(m.faces.data_ptr())
        if atrbvh:
            e = lib.obvh_build_atrbvh_async(V, F, n, flags, a.treelet, 2, 1.2, 1.0, P["nodes"], P["parents"],
                                            P["counts"], P["costs"], P["bounds"], P["obbs"], P["xfs"],
                                            P["collapsed"], P["prims"], W, S)
        else:
            e = lib.obvh_build_async(V, F, n, flags, 1.2, 1.0, P["nodes"], P["parents"], P["counts"], P["costs"],
                                     P["bounds"], P["obbs"], P["xfs"], P["collapsed"], P["prims"], W, S)
        _native.check(e)

    def capture(m):
        """The same build of mesh m as one CUDA graph (obvh_build_graph_create)."""
        h = ctypes.c_void_p()
        V, F = ctypes.c_void_p(m.verts.data_ptr()), ctypes.c_void_p(m.faces.data_ptr())
        if atrbvh:
            e = lib.obvh_build_atrbvh_graph_create(V, F, n, flags, a.treelet, 2, 1.2, 1.0, P["nodes"], P["parents"],
                                                   P["counts"], P["costs"], P["bounds"], P["obbs"], P["xfs"],
                                                   P["collapsed"], P["prims"], W, ctypes.byref(h))
        else:
            e = lib.obvh_build_graph_create(V, F, n, flags, 1.2, 1.0, P["nodes"], P["parents"], P["counts"],
                                            P["costs"], P["bounds"], P["obbs"], P["xfs"], P["collapsed"], P["prims"],
                                            W, ctypes.byref(h))
        _native.check(e)
        return h

    wname = "atrbvh_obb_tree" if atrbvh else "lbvh_obb_tree"
    sampler = ClockSampler(dev.index, enabled=not a.profile)
    if a.profile:
        total_ms, prof, clocks = timed_steps(a, dist, step, sampler, stream)
        return {"profile": wname, "tris": n, "ms_per_step": total_ms / a.steps, "kernels": prof}
    # the timed region: one graph replay per build, no per-launch events
    graphs = [capture(m) for m in meshes]

    def graph_step(j, g=None):
        _native.check(lib.obvh_build_graph_launch(g or graphs[j & 1], S))

    total_ms, _, clocks = timed_steps(a, dist, graph_step, sampler, stream, profile=False)
    # the kernel table: as many builds again, launched one by one with an
    # event pair around every launch (their own timed region)
    kernel_ms, prof, _ = timed_steps(a, dist, step, ClockSampler(dev.index, enabled=False), stream)
    err, slots = ctypes.c_uint32(0), ctypes.c_uint32(0)
    _native.check(status_fn(W, n, S, ctypes.byref(err), ctypes.byref(slots)))
    if err.value != 0:
        raise RuntimeError(f"device error word {err.value}")

    ms_step = total_ms / a.steps
    value = dist.world * nn * a.steps / (total_ms / 1e3) / 1e6
    peak, peak_kind = peaks()
    algo = tree_bytes_per_launch(n)
    # the fused build searches the candidate frames in two launches per step
    # (the nodes completed inside CTA blocks, then those across them): their
    # bytes per step are spread over the launches, so that achieved GB/s is
    # the step's candidate bytes over the step's candidate time
    cl = prof.get("candidate_kernel", (0, 0.0))[0] / a.steps
    if cl > 1:
        algo["candidate_kernel"] = algo["candidate_kernel"] / cl
    kern = kernel_table(prof, a.steps, algo, peak)
    roof = roofline(prof, algo, peak, peak_kind, os.path.join(ROOT, "profiles", f"{wname}_traffic.json"))
    launches = sum(v[0] for v in prof.values())

    # End to end through the C ABI: every step copies its mesh in from pinned
    # host memory, builds, transforms and collapses it, and reads the root box
    # + root cost back to the host.
    pinned = [(torch.from_numpy(v).pin_memory(), torch.from_numpy(bvh.as_faces4(f).view(np.int32)).pin_memory())
              for v, f in host_meshes]
    stagings = [bvh.Mesh(host_meshes[0][0], host_meshes[0][1], device=dev) for _ in range(2)]
    staging_graphs = [capture(m) for m in stagings]
    results = [torch.empty(16, dtype=f32).pin_memory() for _ in range(2)]
    e2e_steps = max(3, min(a.steps, 10))

    def e2e_serial_step(j):
        pv, pf = pinned[j & 1]
        staging, result = stagings[0], results[0]
        staging.verts.copy_(pv, non_blocking=True)
        staging.faces.copy_(pf, non_blocking=True)
        graph_step(j, staging_graphs[0])
        result[:15].copy_(out["obbs"][:15], non_blocking=True)
        result[15:].copy_(out["costs"][:1], non_blocking=True)
        stream.synchronize()

    e2e_serial_step(0)
    t0 = time.perf_counter()
    for j in range(e2e_steps):
        e2e_serial_step(j)
    serial_s = time.perf_counter() - t0

    # Streamed: mesh j+1 is copied in on a second stream while mesh j builds
    # (two staging buffers; a copy waits until the build that last read its
    # buffer is done, a build waits for its copy).
    copy_stream = torch.cuda.Stream(dev)
    h2d_done = [torch.cuda.Event() for _ in range(2)]
    build_done = [torch.cuda.Event() for _ in range(2)]
    read_done = [torch.cuda.Event() for _ in range(2)]
    built = [False, False]

    def issue_copy(j):
        b = j & 1
        pv, pf = pinned[j & 1]
        with torch.cuda.stream(copy_stream):
            if built[b]:
                copy_stream.wait_event(build_done[b])
            stagings[b].verts.copy_(pv, non_blocking=True)
            stagings[b].faces.copy_(pf, non_blocking=True)
            h2d_done[b].record(copy_stream)

    def issue_build(j):
        b = j & 1
        stream.wait_event(h2d_done[b])
        graph_step(j, staging_graphs[b])
        build_done[b].record(stream)
        built[b] = True
        results[b][:15].copy_(out["obbs"][:15], non_blocking=True)
        results[b][15:].copy_(out["costs"][:1], non_blocking=True)
        read_done[b].record(stream)

    def streamed(steps):
        issue_copy(0)
        for j in range(steps):
            if j + 1 < steps:
                issue_copy(j + 1)
            issue_build(j)
            if j >= 1:
                read_done[(j - 1) & 1].synchronize()  # the host has step j-1's result
        read_done[(steps - 1) & 1].synchronize()

    streamed(2)
    t0 = time.perf_counter()
    streamed(e2e_steps)
    e2e_s = time.perf_counter() - t0
    e2e_min = -dist.max(-(nn * e2e_steps / e2e_s / 1e6))
    serial_min = -dist.max(-(nn * e2e_steps / serial_s / 1e6))

    if atrbvh:
        metric = "ATRBVH + OBB-tree + collapse build throughput (Mnodes/s)"
        data = ("synthetic: (2,3) torus-knot tube, 1024 segments x 448 around, radius 0.15, radial bump "
                "0.02 sin(13 theta) cos(7 phi) + U[0,0.005] noise")
        config = {"workload": "atrbvh_obb_tree_collapse", "triangles_per_gpu": n, "nodes_per_gpu": nn,
                  "morton_bits": 63, "treelet_size": a.treelet, "iterations": 2, "ci": 1.2, "ct": 1.0,
                  "l2": "two 26 MB knots alternated; each step writes ~0.6 GB after reading its input, no flush",
                  "parallelism": f"replicas{dist.world}"}
        api = "obvh_build_graph_launch of obvh_build_atrbvh_graph_create (ATRBVH + OBB tree + collapse), pinned host mesh"
    else:
        metric = "LBVH + OBB-tree + collapse build throughput (Mnodes/s)"
        data = "synthetic: thin random triangles (centroid U[0,1]^3, vertex radius log-U[0.002,0.02]), seeded"
        config = {"workload": "lbvh_obb_tree_collapse", "triangles_per_gpu": n, "nodes_per_gpu": nn,
                  "morton_bits": 30, "ci": 1.2, "ct": 1.0,
                  "l2": "two 104 MB meshes alternated between steps; each step writes ~1 GB",
                  "parallelism": f"replicas{dist.world}"}
        api = "obvh_build_graph_launch of obvh_build_graph_create (LBVH + OBB tree + collapse), pinned host mesh"
    line = {
        "metric": metric,
        "value": round(value, 3), "unit": "Mnodes/s", "n_gpus": dist.world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": round(ms_step, 5), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": data, "config": config,
        "launch": "one CUDA graph replay per build (obvh_build_graph_launch); the kernels, their roofline and "
                  "gpu_launches come from as many builds again launched one by one (obvh_build_*async) with an "
                  "event pair around every launch",
        "kernels_pass_ms_per_step": round(kernel_ms / a.steps, 5),
        "kernels": kern, "gpu_launches": launches, "roofline": roof,
        "e2e": {"value": round(dist.world * e2e_min, 3), "unit": "Mnodes/s",
                "h2d_bytes_per_step": int(host_meshes[0][0].nbytes + n * 16), "d2h_bytes_per_step": 64,
                "api": api + "; the copy of mesh j+1 (second stream) overlaps the build of mesh j",
                "serial": {"value": round(dist.world * serial_min, 3),
                           "api": "the same calls with each step's copy, build and read-back waited for in turn"}},
        "clocks": clocks,
    }
    # tree quality of the last build (SAH over the root's area, on the device)
    q = [bvh.bvh_sah(out["nodes"], out["parents"], o).cpu().tolist()[1] for o in (None, out["obbs"])]
    q.append(bvh.bvh_sah(out["collapsed"], out["parents"], out["obbs"]).cpu().tolist()[1])
    line["tree_quality"] = {"sah_aabb": round(q[0], 4), "sah_obb": round(q[1], 4), "sah_obb_collapsed": round(q[2], 4),
                            "ci": 1.2, "ct": 1.0, "api": "obvh_bvh_sah_async (kr_bvh_sah's cost, on the device)"}
    torch.cuda.synchronize()
    for g in graphs + staging_graphs:
        _native.check(lib.obvh_build_graph_destroy(g))
    if dist.rank == 0 and dist.world == 1:
        line["cpu_baseline"] = cpu_atrbvh_baseline(a.treelet) if atrbvh else cpu_tree_baseline()
    return line


def cpu_tree_baseline(n=200_000):
    """The oracle port of the same build on one host core (the reference has
    no CPU implementation of this GPU path)."""
    from oracle import bvh as ref
    from obvh_b200 import workloads
    v, f = workloads.triangle_soup(n, seed=77)
    reps, t0 = 0, time.perf_counter()
    while True:
        r = ref.lbvh_build(v, f)
        ref.obb_tree(r["nodes"], r["parents"], v, f)
        ref.collapse(r["nodes"], r["parents"], r["counts"], r["costs"])
        reps += 1
        dt = time.perf_counter() - t0
        if dt > 8.0 or reps >= 20:
            break
    return {"value": round((2 * n - 1) * reps / dt / 1e6, 4), "unit": "Mnodes/s", "cores": 1, "kind": "port",
            "sample": f"{reps} builds of {n} triangles ({dt:.1f} s), oracle C restatement"}


def _atrbvh_port_build(v, f, tau):
    from oracle import bvh as ref
    r = ref.atrbvh_build(v, f, tau, 2)
    ref.obb_tree(r["nodes"], r["parents"], v, f)
    ref.collapse(r["nodes"], r["parents"], r["counts"], r["costs"])


def cpu_atrbvh_baseline(tau, segments=256, around=112):
    """The oracle port of the ATRBVH commit on one host core, on a smaller
    knot of the same shape (the reference has no CPU implementation)."""
    from obvh_b200 import workloads
    v, f = workloads.torus_knot_mesh(segments, around, seed=77)
    n = f.shape[0]
    reps, t0 = 0, time.perf_counter()
    while True:
        _atrbvh_port_build(v, f, tau)
        reps += 1
        dt = time.perf_counter() - t0
        if dt > 8.0 or reps >= 20:
            break
    return {"value": round((2 * n - 1) * reps / dt / 1e6, 4), "unit": "Mnodes/s", "cores": 1, "kind": "port",
            "sample": f"{reps} builds of a {n}-triangle knot ({segments}x{around}, {dt:.1f} s), oracle C restatement"}


def bench_atrbvh_reference(a, dist):
    """The CPU restatement of the ATRBVH commit (oracle port) on this host's
    cores, on a bounded knot of the benchmark's shape: each step, every host
    thread builds its own copy."""
    from obvh_b200 import workloads
    segments, around = 256, 112
    v, f = workloads.torus_knot_mesh(segments, around, seed=2)
    n = f.shape[0]
    threads = host_threads()
    times = parallel_steps(a, lambda: _atrbvh_port_build(v, f, a.treelet), threads)
    value = threads * (2 * n - 1) * len(times) / sum(times) / 1e6
    return {"metric": "ATRBVH + OBB-tree + collapse build throughput (Mnodes/s)", "impl": "reference",
            "value": round(value, 4), "unit": "Mnodes/s", "n_gpus": dist.world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(1e3 * sum(times) / len(times), 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (same generator as the ours arm)",
            "config": {"workload": "atrbvh_obb_tree_collapse", "treelet_size": a.treelet, "iterations": 2,
                       "sample_triangles": n},
            "cpu_baseline": {"value": round(value, 4), "unit": "Mnodes/s", "cores": threads, "kind": "port",
                             "sample": f"{threads} concurrent builds of a {segments}x{around} knot ({n} triangles) "
                                       "per step, oracle C restatement"},
            "e2e": {"value": round(value, 4), "unit": "Mnodes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def host_threads(cap=64):
    """Host threads this process may use (capped: every thread holds a sample
    build's working memory)."""
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    return max(1, min(n, cap))


def parallel_steps(a, work, threads):
    """Times steps in which `threads` host threads each run work() once
    (the oracle's C calls release the GIL); returns the timed steps' seconds."""
    from concurrent.futures import ThreadPoolExecutor
    times = []
    with ThreadPoolExecutor(max_workers=threads) as pool:
        for j in range(a.warmup + a.steps):
            t0 = time.perf_counter()
            list(pool.map(lambda _: work(), range(threads)))
            if j >= a.warmup:
                times.append(time.perf_counter() - t0)
    return times


def bench_tree_reference(a, dist):
    """The CPU restatement of the path (oracle port) on this host's cores: the
    reference has no CPU implementation of its GPU build to run.  Each step,
    every host thread builds its own copy of a sample mesh."""
    from oracle import bvh as ref
    from obvh_b200 import workloads
    n = min(a.tris, 200_000)
    v, f = workloads.triangle_soup(n, seed=1)
    threads = host_threads()

    def work():
        r = ref.lbvh_build(v, f)
        ref.obb_tree(r["nodes"], r["parents"], v, f)
        ref.collapse(r["nodes"], r["parents"], r["counts"], r["costs"])

    times = parallel_steps(a, work, threads)
    nn = 2 * n - 1
    value = threads * nn * len(times) / sum(times) / 1e6
    return {"metric": "LBVH + OBB-tree + collapse build throughput (Mnodes/s)", "impl": "reference",
            "value": round(value, 4), "unit": "Mnodes/s", "n_gpus": dist.world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(1e3 * sum(times) / len(times), 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (same generator as the ours arm)",
            "config": {"workload": "lbvh_obb_tree_collapse", "triangles_per_gpu": a.tris, "sample_triangles": n},
            "cpu_baseline": {"value": round(value, 4), "unit": "Mnodes/s", "cores": threads, "kind": "port",
                             "sample": f"{threads} concurrent {n}-triangle builds per step (oracle C restatement, "
                                       "one host thread each)"},
            "e2e": {"value": round(value, 4), "unit": "Mnodes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ---------------------------------------------------------------------------
def pack_bytes(nodes):
    """Algorithmic bytes of one fused packing pass (pack_kernel) over a tree:
    every node read (36 B) and its metadata word read and written (16 + 16 B);
    an internal node also reads both children's boxes and counts (2 x 28 B)
    and transforms (2 x 64 B) and writes its record (60 B), its pair (128 B)
    and two 4x3 rows (96 B); a node with primitives writes 36 B of its record;
    an internal-index node without a new pair reads the pair (128 B) for its
    SoA rows (96 B)."""
    import numpy as np
    npr = nodes["n_prims"].astype(np.int64)
    nn = npr.shape[0]
    ni = (nn - 1) // 2
    internal = npr == 0
    leafy = (npr != 0) & (npr != 0xFFFF)
    no_pair = ~internal & (np.arange(nn) < ni)
    return int(68 * nn + internal.sum() * (56 + 128 + 60 + 128 + 96) + leafy.sum() * 36 + no_pair.sum() * (128 + 96))


def _pack_tree(n, seed, dev):
    """The collapsed tree and OBB transforms of an n-triangle fused build (device)."""
    import torch
    from obvh_b200 import bvh, workloads
    v, f = workloads.triangle_soup(n, seed=seed)
    b = bvh.ObvhBuilder(dev)
    o = b.build(bvh.Mesh(v, f, device=dev), flags=3)
    torch.cuda.synchronize()
    if b.status(n)[0]:
        raise RuntimeError("build failed")
    return o["collapsed"].clone(), o["transforms"].clone()


def bench_pack_ours(a, dist):
    """Traversal packing of the collapsed OBB tree of the 2M-triangle soup:
    packed records, child-transform pairs and SoA OBVH arrays in one pass."""
    import ctypes as c
    import torch
    from obvh_b200 import _native, bvh
    n = a.tris
    dev = torch.device("cuda", torch.cuda.current_device())
    nodes, xfs = _pack_tree(n, 1 + dist.rank, dev)
    nn, ni = 2 * n - 1, n - 1
    out = {"packed": torch.zeros(nn * 64, dtype=torch.uint8, device=dev),
           "pairs": torch.zeros(ni * 32, dtype=torch.float32, device=dev),
           "left_T": torch.zeros(ni * 12, dtype=torch.float32, device=dev),
           "right_T": torch.zeros(ni * 12, dtype=torch.float32, device=dev),
           "metadata": torch.zeros(nn * 4, dtype=torch.int32, device=dev),
           "error": torch.zeros(1, dtype=torch.int32, device=dev)}
    lib = _native.lib()
    stream = torch.cuda.current_stream(dev)
    ptr = {k: c.c_void_p(t.data_ptr()) for k, t in out.items()}
    s_ptr = c.c_void_p(stream.cuda_stream)

    def step(j):
        _native.check(lib.obvh_obvh_pack_async(c.c_void_p(nodes.data_ptr()), c.c_void_p(xfs.data_ptr()),
                                               ptr["packed"], ptr["pairs"], ptr["left_T"], ptr["right_T"],
                                               ptr["metadata"], nn, ni, ptr["error"], s_ptr))

    sampler = ClockSampler(dev.index, enabled=not a.profile)
    total_ms, prof, clocks = timed_steps(a, dist, step, sampler, stream)
    if int(out["error"].item()):
        raise RuntimeError("packing reported a malformed tree")
    if a.profile:
        return {"profile": "obvh_pack", "triangles": n, "ms_per_step": total_ms / a.steps, "kernels": prof}
    nodes_np = bvh.nodes_numpy(nodes)
    algo = {"pack_kernel": pack_bytes(nodes_np)}
    peak, peak_kind = peaks()
    value = dist.world * nn * a.steps / (total_ms / 1e3) / 1e6
    roof = roofline(prof, algo, peak, peak_kind, os.path.join(ROOT, "profiles", "obvh_pack_traffic.json"))

    # end to end through the reference-facing calls: the tree and transforms
    # copied from pinned host memory, kr_cuda_obvh_persistent, then
    # kr_cuda_soa_obvh with its arrays read back to the host
    h_nodes = torch.empty(nodes.shape, dtype=nodes.dtype, pin_memory=True)
    h_xfs = torch.empty(xfs.shape, dtype=xfs.dtype, pin_memory=True)
    h_nodes.copy_(nodes)
    h_xfs.copy_(xfs)
    d_nodes, d_xfs = torch.empty_like(nodes), torch.empty_like(xfs)
    h_soa = {"left_T": torch.empty(ni * 12, dtype=torch.float32, pin_memory=True),
             "right_T": torch.empty(ni * 12, dtype=torch.float32, pin_memory=True),
             "metadata": torch.empty(nn * 4, dtype=torch.int32, pin_memory=True)}

    def e2e_step():
        d_nodes.copy_(h_nodes, non_blocking=True)
        d_xfs.copy_(h_xfs, non_blocking=True)
        torch.cuda.synchronize()
        o = bvh.persistent(d_nodes, nn, d_xfs, out["packed"], out["pairs"])
        bvh.soa_obvh(o["packed"], o["pairs"], ni, nn, out=h_soa)

    e2e_step()
    e2e_steps = max(3, min(a.steps, 10))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    e2e_s = time.perf_counter() - t0
    e2e_min = -dist.max(-(nn * e2e_steps / e2e_s / 1e6))
    line = {
        "metric": "OBVH traversal packing throughput (Mnodes/s)", "value": round(value, 3), "unit": "Mnodes/s",
        "n_gpus": dist.world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(total_ms / a.steps, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: collapsed LBVH OBB tree of the 2M thin-triangle soup (same generator as lbvh_obb_tree)",
        "config": {"workload": "obvh_pack_collapsed_tree", "triangles_per_gpu": n, "nodes_per_gpu": nn,
                   "l2": "inputs 400 MB and outputs 768 MB per pass (> 126 MB L2), no flush",
                   "parallelism": f"replicas{dist.world}"},
        "kernels": kernel_table(prof, a.steps, algo, peak),
        "gpu_launches": sum(v[0] for v in prof.values()), "roofline": roof,
        "e2e": {"value": round(dist.world * e2e_min, 3), "unit": "Mnodes/s",
                "h2d_bytes_per_step": nn * (36 + 64), "d2h_bytes_per_step": ni * 96 + nn * 16,
                "api": "kr_cuda_obvh_persistent + kr_cuda_soa_obvh, tree from pinned host memory, SoA read back "
                       "into pinned host memory"},
        "clocks": clocks,
    }
    if dist.rank == 0 and dist.world == 1:
        from oracle import bvh as ref
        xf_np = xfs.cpu().numpy().reshape(-1, 16)
        reps, t0 = 0, time.perf_counter()
        while True:
            pk, pr = ref.pack(nodes_np, xf_np)
            ref.soa_obvh(pk, pr, ni)
            reps += 1
            dt = time.perf_counter() - t0
            if dt > 8.0 or reps >= 10:
                break
        line["cpu_baseline"] = {"value": round(nn * reps / dt / 1e6, 3), "unit": "Mnodes/s", "cores": 1,
                                "kind": "port",
                                "sample": f"{reps} packings of the same {nn}-node tree ({dt:.1f} s), oracle C "
                                          "restatement"}
    return line


def bench_pack_reference(a, dist):
    """The CPU restatement of the packing (oracle port) on this host's cores,
    on the collapsed tree of a 200K-triangle sample: every host thread packs
    its own copy each step (the reference packs on the GPU and converts to SoA
    through a single-threaded host loop)."""
    from oracle import bvh as ref
    from obvh_b200 import workloads
    n = min(a.tris, 200_000)
    v, f = workloads.triangle_soup(n, seed=1)
    r = ref.lbvh_build(v, f)
    _, xfs, _ = ref.obb_tree(r["nodes"], r["parents"], v, f)
    col, _, _, _, _ = ref.collapse(r["nodes"], r["parents"], r["counts"], r["costs"])
    threads = host_threads()
    nn = 2 * n - 1

    def work():
        pk, pr = ref.pack(col, xfs)
        ref.soa_obvh(pk, pr, n - 1)

    times = parallel_steps(a, work, threads)
    value = threads * nn * len(times) / sum(times) / 1e6
    return {"metric": "OBVH traversal packing throughput (Mnodes/s)", "impl": "reference",
            "value": round(value, 4), "unit": "Mnodes/s", "n_gpus": dist.world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(1e3 * sum(times) / len(times), 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (same generator as the ours arm)",
            "config": {"workload": "obvh_pack_collapsed_tree", "triangles_per_gpu": a.tris, "sample_triangles": n},
            "cpu_baseline": {"value": round(value, 4), "unit": "Mnodes/s", "cores": threads, "kind": "port",
                             "sample": f"{threads} concurrent packings of a {n}-triangle collapsed tree per step "
                                       "(oracle C restatement, one host thread each)"},
            "e2e": {"value": round(value, 4), "unit": "Mnodes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ---------------------------------------------------------------------------
def trace_bytes_per_ray(counts, hit_fraction):
    """Bytes a traversal touches per ray (read once each, cached or not): the
    ray (32 B) and its record (28 B), per internal node its metadata and two
    4x3 rows (16 + 96 B), per leaf its metadata (16 B), per triangle tested
    its face and vertices (16 + 36 B), per primitive-list entry 4 B, and per
    hit the hit triangle again for the normal (52 B)."""
    return (60 + 112 * counts["internal_visits"] + 16 * counts["leaf_visits"] + 52 * counts["triangle_tests"]
            + 4 * counts["list_reads"] + 52 * hit_fraction)


def _trace_scene(n, dev):
    """The collapsed OBB tree of the n-triangle soup packed as a SoA OBVH (device)."""
    import torch
    from obvh_b200 import bvh, workloads
    v, f = workloads.triangle_soup(n, seed=1)
    mesh = bvh.Mesh(v, f, device=dev)
    b = bvh.ObvhBuilder(dev)
    o = b.build(mesh, flags=3)
    torch.cuda.synchronize()
    if b.status(n)[0]:
        raise RuntimeError("build failed")
    s = bvh.obvh_pack(o["collapsed"], 2 * n - 1, n - 1, o["transforms"])
    torch.cuda.synchronize()
    return v, f, mesh, s, o["primitives"], o


def bench_trace_ours(a, dist):
    """Closest-hit traversal of a.rays probe rays through the SoA OBVH of the
    collapsed 2M-triangle soup tree."""
    import ctypes as c
    import numpy as np
    import torch
    from obvh_b200 import _native, bvh, workloads
    n = a.tris
    dev = torch.device("cuda", torch.cuda.current_device())
    v, f, mesh, soa, prims, _ = _trace_scene(n, dev)
    nn, ni = 2 * n - 1, n - 1
    ray_sets = [workloads.probe_rays(a.rays, [0, 0, 0], [1, 1, 1], seed=21 + 2 * dist.rank + j) for j in range(2)]
    d_rays = [torch.from_numpy(r.view(np.uint8).copy()).to(dev) for r in ray_sets]
    isects = torch.empty(28 * a.rays, dtype=torch.uint8, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    lib = _native.lib()
    stream = torch.cuda.current_stream(dev)
    P = lambda t: c.c_void_p(t.data_ptr())  # noqa: E731

    def step(j):
        _native.check(lib.obvh_soa_obvh_intersect_async(P(soa["left_T"]), P(soa["right_T"]), P(soa["metadata"]), ni,
                                                        nn, P(mesh.verts), P(mesh.faces), n, P(prims), prims.numel(),
                                                        P(d_rays[j & 1]), P(isects), a.rays, P(err),
                                                        c.c_void_p(stream.cuda_stream)))

    sampler = ClockSampler(dev.index, enabled=not a.profile)
    total_ms, prof, clocks = timed_steps(a, dist, step, sampler, stream)
    if int(err.item()):
        raise RuntimeError("traversal reported a bad index")
    if a.profile:
        return {"profile": "obvh_trace", "rays": a.rays, "ms_per_step": total_ms / a.steps, "kernels": prof}
    hits = np.frombuffer(isects.cpu().numpy().tobytes(), dtype=workloads.ISECT)
    hit_fraction = float((hits["primitive"] != 0xFFFFFFFF).mean())
    peak, peak_kind = peaks()
    value = dist.world * a.rays * a.steps / (total_ms / 1e3) / 1e6

    # work per ray from the oracle's counters on a sample of the same rays
    from oracle import bvh as ref
    lt = soa["left_T"].cpu().numpy().reshape(-1, 12)[:ni]
    rt = soa["right_T"].cpu().numpy().reshape(-1, 12)[:ni]
    meta = soa["metadata"].cpu().numpy().reshape(-1, 4)
    pr = prims.cpu().numpy().view(np.uint32)
    counts = ref.soa_obvh_traversal_counts(lt, rt, meta, v, f, pr, ray_sets[0][:20_000])
    per_ray = trace_bytes_per_ray(counts, hit_fraction)
    algo = {"trace_kernel": int(per_ray * a.rays)}
    roof = roofline(prof, algo, peak, peak_kind, os.path.join(ROOT, "profiles", "obvh_trace_traffic.json"))

    # end to end through kr_cuda_soa_obvh_intersect: the scene resident, the
    # rays copied from pinned host memory and the records read back each step
    d_soa = c.c_void_p(0)
    _native.check(lib.kr_cuda_soa_obvh(P(soa["packed"]), P(soa["pairs"]), c.byref(d_soa), ni, nn))
    h_rays = torch.empty(32 * a.rays, dtype=torch.uint8, pin_memory=True)
    h_rays.copy_(d_rays[0])
    h_isects = torch.empty(28 * a.rays, dtype=torch.uint8, pin_memory=True)
    counter = torch.zeros(1, dtype=torch.int32, device=dev)

    def e2e_step():
        d_rays[1].copy_(h_rays, non_blocking=True)
        torch.cuda.synchronize()
        _native.check(lib.kr_cuda_soa_obvh_intersect(d_soa, P(mesh.verts), P(mesh.faces), P(prims), P(d_rays[1]),
                                                     P(isects), a.rays, 128, 0, P(counter)))
        h_isects.copy_(isects)

    try:
        e2e_step()
        e2e_steps = max(3, min(a.steps, 10))
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            e2e_step()
        e2e_s = time.perf_counter() - t0
    finally:
        _native.check(lib.obvh_soa_obvh_free(d_soa))
    e2e_min = -dist.max(-(a.rays * e2e_steps / e2e_s / 1e6))
    line = {
        "metric": "OBVH closest-hit traversal throughput (Mrays/s)", "value": round(value, 3), "unit": "Mrays/s",
        "n_gpus": dist.world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(total_ms / a.steps, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: probe rays from a sphere around [0,1]^3 towards uniform points in it, through the "
                "collapsed OBB tree of the 2M thin-triangle soup",
        "config": {"workload": "obvh_trace_collapsed_tree", "triangles": n, "rays_per_gpu": a.rays,
                   "hit_fraction": round(hit_fraction, 4), "work_per_ray": {k: round(x, 2) for k, x in counts.items()},
                   "l2": "two ray sets of 128 MB alternated; the tree's SoA (256 MB) and mesh (104 MB) exceed L2",
                   "parallelism": f"replicas{dist.world}"},
        "kernels": kernel_table(prof, a.steps, algo, peak),
        "gpu_launches": sum(x[0] for x in prof.values()), "roofline": roof,
        "e2e": {"value": round(dist.world * e2e_min, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 32 * a.rays,
                "d2h_bytes_per_step": 28 * a.rays,
                "api": "kr_cuda_soa_obvh_intersect, rays from pinned host memory, records read back to pinned memory"},
        "clocks": clocks,
    }
    if dist.rank == 0 and dist.world == 1:
        sample = ray_sets[0][:200_000]
        t0 = time.perf_counter()
        ref.soa_obvh_intersect(lt, rt, meta, v, f, pr, sample, threads=1)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": round(len(sample) / dt / 1e6, 4), "unit": "Mrays/s", "cores": 1,
                                "kind": "port",
                                "sample": f"{len(sample)} of the rays ({dt:.1f} s), oracle C restatement"}
    return line


def bench_trace_compressed_ours(a, dist):
    """Closest-hit traversal of a.rays probe rays through the compressed SoA
    OBVH (24-byte boxes per child, quantised frames) of the collapsed
    2M-triangle soup tree, beside the SoA OBVH traversal on the same rays."""
    import ctypes as c
    import numpy as np
    import torch
    from obvh_b200 import _native, bvh, workloads
    n = a.tris
    dev = torch.device("cuda", torch.cuda.current_device())
    v, f, mesh, soa, prims, o = _trace_scene(n, dev)
    nn, ni = 2 * n - 1, n - 1
    pairs = bvh.compressed_pairs_from_obbs(bvh.nodes_numpy(o["collapsed"]), o["obbs"].cpu().numpy())
    d_pairs = torch.from_numpy(pairs).to(dev)
    comp = bvh.soa_compressed_obvh(soa["packed"], d_pairs, ni, nn)
    torch.cuda.synchronize()
    ray_sets = [workloads.probe_rays(a.rays, [0, 0, 0], [1, 1, 1], seed=21 + 2 * dist.rank + j) for j in range(2)]
    d_rays = [torch.from_numpy(r.view(np.uint8).copy()).to(dev) for r in ray_sets]
    isects = torch.empty(28 * a.rays, dtype=torch.uint8, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    lib = _native.lib()
    stream = torch.cuda.current_stream(dev)
    P = lambda t: c.c_void_p(t.data_ptr())  # noqa: E731

    def step(j):
        _native.check(lib.obvh_soa_compressed_obvh_intersect_async(
            P(comp["lbounds"]), P(comp["rbounds"]), P(comp["metadata"]), ni, nn, P(mesh.verts), P(mesh.faces), n,
            P(prims), prims.numel(), P(d_rays[j & 1]), P(isects), a.rays, P(err), c.c_void_p(stream.cuda_stream)))

    def step_soa(j):
        _native.check(lib.obvh_soa_obvh_intersect_async(P(soa["left_T"]), P(soa["right_T"]), P(soa["metadata"]), ni,
                                                        nn, P(mesh.verts), P(mesh.faces), n, P(prims), prims.numel(),
                                                        P(d_rays[j & 1]), P(isects), a.rays, P(err),
                                                        c.c_void_p(stream.cuda_stream)))

    sampler = ClockSampler(dev.index, enabled=not a.profile)
    total_ms, prof, clocks = timed_steps(a, dist, step, sampler, stream)
    if int(err.item()):
        raise RuntimeError("compressed traversal reported a bad index")
    if a.profile:
        return {"profile": "obvh_trace_compressed", "rays": a.rays, "ms_per_step": total_ms / a.steps,
                "kernels": prof}
    hits = np.frombuffer(isects.cpu().numpy().tobytes(), dtype=workloads.ISECT)
    hit_fraction = float((hits["primitive"] != 0xFFFFFFFF).mean())
    value = dist.world * a.rays * a.steps / (total_ms / 1e3) / 1e6
    soa_ms, _, _ = timed_steps(a, dist, step_soa, ClockSampler(dev.index, enabled=False), stream)
    soa_value = dist.world * a.rays * a.steps / (soa_ms / 1e3) / 1e6
    exact = np.frombuffer(isects.cpu().numpy().tobytes(), dtype=workloads.ISECT)
    exact_hits = float((exact["primitive"] != 0xFFFFFFFF).mean())
    node_bytes = {"compressed": 48 * ni + 16 * nn, "soa_obvh": 96 * ni + 16 * nn}

    # end to end through kr_cuda_soa_compressed_obvh + kr_cuda_obvh_compressed_persistent_intersect:
    # the scene resident, the rays copied from pinned host memory and the records read back each step
    d_soa = c.c_void_p(0)
    _native.check(lib.kr_cuda_soa_compressed_obvh(P(soa["packed"]), P(d_pairs), c.byref(d_soa), ni, nn))
    h_rays = torch.empty(32 * a.rays, dtype=torch.uint8, pin_memory=True)
    h_rays.copy_(d_rays[0])
    h_isects = torch.empty(28 * a.rays, dtype=torch.uint8, pin_memory=True)
    counter = torch.zeros(1, dtype=torch.int32, device=dev)

    def e2e_step():
        d_rays[1].copy_(h_rays, non_blocking=True)
        torch.cuda.synchronize()
        _native.check(lib.kr_cuda_obvh_compressed_persistent_intersect(d_soa, P(mesh.verts), P(mesh.faces), P(prims),
                                                                       P(d_rays[1]), P(isects), a.rays, 128, 0,
                                                                       P(counter)))
        h_isects.copy_(isects)

    try:
        e2e_step()
        e2e_steps = max(3, min(a.steps, 10))
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            e2e_step()
        e2e_s = time.perf_counter() - t0
    finally:
        _native.check(lib.obvh_soa_obvh_compressed_free(d_soa))
    e2e_min = -dist.max(-(a.rays * e2e_steps / e2e_s / 1e6))
    peak, peak_kind = peaks()
    name, (launches, kms) = max(prof.items(), key=lambda kv: kv[1][1])
    return {
        "metric": "Compressed OBVH closest-hit traversal throughput (Mrays/s)", "value": round(value, 3),
        "unit": "Mrays/s", "n_gpus": dist.world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": round(total_ms / a.steps, 5), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: probe rays from a sphere around [0,1]^3 towards uniform points in it, through the "
                "compressed form of the collapsed OBB tree of the 2M thin-triangle soup (pairs from the tree's "
                "own boxes, obvh_b200.bvh.compressed_pairs_from_obbs)",
        "config": {"workload": "obvh_trace_compressed_collapsed_tree", "triangles": n, "rays_per_gpu": a.rays,
                   "hit_fraction": round(hit_fraction, 4), "hit_fraction_soa_obvh": round(exact_hits, 4),
                   "node_array_bytes": node_bytes,
                   "l2": "two ray sets of 128 MB alternated; node arrays and mesh exceed L2",
                   "parallelism": f"replicas{dist.world}"},
        "kernels": kernel_table(prof, a.steps, {}, peak), "gpu_launches": sum(x[0] for x in prof.values()),
        "roofline": {"bound": "hbm", "kernel": name, "achieved": None, "peak": peak, "unit": "GB/s", "frac": None,
                     "traffic": None, "peak_source": peak_kind, "launches": launches,
                     "ms_per_launch": round(kms / max(launches, 1), 5),
                     "note": "work per ray (node and triangle fetches) is not counted for the compressed form"},
        "soa_obvh": {"value": round(soa_value, 3), "unit": "Mrays/s", "ms_per_step": round(soa_ms / a.steps, 5),
                     "api": "obvh_soa_obvh_intersect_async on the same tree and rays"},
        "e2e": {"value": round(dist.world * e2e_min, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 32 * a.rays,
                "d2h_bytes_per_step": 28 * a.rays,
                "api": "kr_cuda_obvh_compressed_persistent_intersect, rays from pinned host memory, records read "
                       "back to pinned memory"},
        "clocks": clocks,
    }


def bench_trace_reference(a, dist):
    """The CPU restatement of the traversal (oracle port) on this host's cores:
    each step every host thread traces its slice of a 400K-ray sample through
    the collapsed OBB tree of the 2M-triangle soup (built once, by the oracle)."""
    import numpy as np
    from oracle import bvh as ref
    from obvh_b200 import workloads
    n = a.tris
    v, f = workloads.triangle_soup(n, seed=1)
    r = ref.lbvh_build(v, f)
    _, xfs, _ = ref.obb_tree(r["nodes"], r["parents"], v, f)
    col, _, prims, _, _ = ref.collapse(r["nodes"], r["parents"], r["counts"], r["costs"])
    pk, pr = ref.pack(col, xfs)
    lt, rt, meta = ref.soa_obvh(pk, pr, n - 1)
    rays = workloads.probe_rays(min(a.rays, 400_000), [0, 0, 0], [1, 1, 1], seed=21)
    threads = host_threads()
    times = []
    for j in range(a.warmup + a.steps):
        t0 = time.perf_counter()
        ref.soa_obvh_intersect(lt, rt, meta, v, f, prims, rays, threads=threads)
        if j >= a.warmup:
            times.append(time.perf_counter() - t0)
    value = len(rays) * len(times) / sum(times) / 1e6
    return {"metric": "OBVH closest-hit traversal throughput (Mrays/s)", "impl": "reference",
            "value": round(value, 4), "unit": "Mrays/s", "n_gpus": dist.world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(1e3 * sum(times) / len(times), 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (same generator as the ours arm)",
            "config": {"workload": "obvh_trace_collapsed_tree", "triangles": n, "sample_rays": len(rays)},
            "cpu_baseline": {"value": round(value, 4), "unit": "Mrays/s", "cores": threads, "kind": "port",
                             "sample": f"{len(rays)} rays per step over {threads} host threads (oracle C "
                                       "restatement)"},
            "e2e": {"value": round(value, 4), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ---------------------------------------------------------------------------
def bench_dito_ours(a, dist):
    import torch
    from obvh_b200 import DitoFitter, points_obb, workloads

    n = a.points
    dev = torch.device("cuda", torch.cuda.current_device())
    # two independent point sets alternated between steps (1.2 GB each > 126 MB L2)
    sets = [workloads.ellipsoid_points_torch(n, seed=1234 + 2 * dist.rank + j, device=dev) for j in range(2)]
    fitter = DitoFitter(dev)
    out = torch.empty(15, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    sampler = ClockSampler(dev.index, enabled=not a.profile)
    total_ms, prof, clocks = timed_steps(a, dist, lambda j: fitter.fit(sets[j & 1], out), sampler, stream)
    path, _, err = fitter.report()
    if err:
        raise RuntimeError(f"device error word {err}")
    if a.profile:
        return {"profile": "dito", "points": n, "ms_per_step": total_ms / a.steps, "kernels": prof}
    peak, peak_kind = peaks()
    value = dist.world * n * a.steps / (total_ms / 1e3) / 1e6
    dito_bytes = {"dito_extremal_pass": 12 * n, "dito_extent_pass": 12 * n}
    roof = roofline(prof, dito_bytes, peak, peak_kind, os.path.join(ROOT, "profiles", "dito_traffic.json"))

    host = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
    host.copy_(sets[0])
    host_np = host.numpy()
    points_obb(host_np)
    e2e_steps = max(3, min(a.steps, 10))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        points_obb(host_np)
    e2e_s = time.perf_counter() - t0
    e2e_min = -dist.max(-(n * e2e_steps / e2e_s / 1e6))
    line = {
        "metric": "DiTO-14 fit throughput (Mpoints/s)", "value": round(value, 3), "unit": "Mpoints/s",
        "n_gpus": dist.world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(total_ms / a.steps, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: ellipsoid surface points (4,1,0.25), Haar rotation, N(0,0.01^2) noise, U[-10,10]^3 offset",
        "config": {"workload": "dito_plain_fit", "points_per_gpu": n, "point_bytes": 12,
                   "l2": "two 1.2 GB point sets alternated between steps (> 126 MB L2), no flush",
                   "parallelism": f"replicas{dist.world}", "path": path},
        "kernels": kernel_table(prof, a.steps, dito_bytes, peak),
        "gpu_launches": sum(v[0] for v in prof.values()), "roofline": roof,
        "e2e": {"value": round(dist.world * e2e_min, 3), "unit": "Mpoints/s", "h2d_bytes_per_step": 12 * n,
                "d2h_bytes_per_step": 316, "api": "obvh_points_obb (kr_cuda_points_obb with errors), pinned host"},
        "clocks": clocks,
    }
    if dist.rank == 0 and dist.world == 1:
        import oracle
        oracle.ref_dito14(host_np[:1000])
        t0 = time.perf_counter()
        for _ in range(3):
            oracle.ref_dito14(host_np)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": round(3 * n / dt / 1e6, 3), "unit": "Mpoints/s", "cores": 1,
                                "kind": "reference",
                                "sample": f"3 fits of the {n}-point set ({dt:.1f} s), reference DiTO_14 (oracle/_ref)"}
    return line


def bench_dito_reference(a, dist):
    """The reference's own CPU DiTO_14 (single-threaded, as shipped), one fit per host thread."""
    import numpy as np
    import oracle
    from obvh_b200 import workloads
    n = a.points
    try:
        import torch
        host = workloads.ellipsoid_points_torch(n, seed=1234, device="cuda" if torch.cuda.is_available() else "cpu")
        host = host.cpu().numpy()
    except Exception:
        host = workloads.ellipsoid_points(n, seed=1234)
    host = np.ascontiguousarray(host, dtype=np.float32)
    # every host thread fits the (shared, read-only) set: DiTO_14 itself is single-threaded
    threads = host_threads()
    times = parallel_steps(a, lambda: oracle.ref_dito14(host), threads)
    value = threads * n * len(times) / sum(times) / 1e6
    return {"metric": "DiTO-14 fit throughput (Mpoints/s)", "impl": "reference", "value": round(value, 3),
            "unit": "Mpoints/s", "n_gpus": dist.world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": round(1e3 * sum(times) / len(times), 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (same generator as the ours arm)",
            "config": {"workload": "dito_plain_fit", "points_per_gpu": n},
            "cpu_baseline": {"value": round(value, 3), "unit": "Mpoints/s", "cores": threads, "kind": "reference",
                             "sample": f"{threads} concurrent full {n}-point fits per step (DiTO_14<float> is "
                                       "single-threaded; one fit per host thread)"},
            "e2e": {"value": round(value, 3), "unit": "Mpoints/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def bench_batch_ours(a, dist):
    import numpy as np
    import torch
    from obvh_b200 import _native, workloads
    from obvh_b200.batch import DitoBatch, points_obb_batch

    dev = torch.device("cuda", torch.cuda.current_device())
    pts, offsets = workloads.gaussian_sets_torch(a.sets, seed=3 + dist.rank, device=dev)
    total = int(offsets[-1])
    out = torch.empty((a.sets, 15), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    batch = DitoBatch(offsets)
    tuning, tuned_ms = (batch.tuning, None) if (a.no_autotune or a.profile) else batch.autotune(pts, out, repeats=3)
    batch.capture(pts, out)
    sampler = ClockSampler(dev.index, enabled=not a.profile)
    total_ms, prof, clocks = timed_steps(a, dist, lambda j: batch.launch(stream), sampler, stream)
    if batch.status(stream):
        raise RuntimeError("device error word set")
    if a.profile:
        return {"profile": "dito_batch", "sets": a.sets, "points": total, "ms_per_step": total_ms / a.steps,
                "kernels": prof}
    peak, peak_kind = peaks()
    value = dist.world * total * a.steps / (total_ms / 1e3) / 1e6
    # every set (at most 3 MB) fits in L2 between its two passes: 12 B/point compulsory
    batch_bytes = {"dito_batch_kernel": 12 * total}
    roof = roofline(prof, batch_bytes, peak, peak_kind,
                    os.path.join(ROOT, "profiles", "dito_batch_traffic.json"))

    # plain per-call path on the same device-resident buffer: one fit per set
    lib = _native.lib()
    ws = torch.zeros(int(lib.obvh_dito_workspace_bytes()), dtype=torch.uint8, device=dev)
    W, S = ctypes.c_void_p(ws.data_ptr()), ctypes.c_void_p(stream.cuda_stream)
    base, obase = pts.data_ptr(), out.data_ptr()
    calls = [(ctypes.c_void_p(base + 12 * int(offsets[s])), int(offsets[s + 1] - offsets[s]),
              ctypes.c_void_p(obase + 60 * s)) for s in range(a.sets)]

    def per_call(st):
        for p, n, o in calls:
            e = lib.obvh_dito_fit_async(p, n, 0, o, W, st)
            if e:
                _native.check(e)
    per_call(S)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 2
    e0.record(stream)
    for _ in range(reps):
        per_call(S)
    e1.record(stream)
    torch.cuda.synchronize()
    host_loop_ms = e0.elapsed_time(e1) / reps
    # the same per-set launches captured once into a CUDA graph and replayed:
    # the per-call path without the host's launch overhead, i.e. what the
    # device itself spends on one fit per call
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        per_call(ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    g.replay()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        g.replay()
    e1.record(stream)
    torch.cuda.synchronize()
    pc_ms = e0.elapsed_time(e1) / reps
    del g
    pc_value = -dist.max(-(total / (pc_ms / 1e3) / 1e6)) * dist.world

    host = torch.empty((total, 3), dtype=torch.float32, pin_memory=True)
    host.copy_(pts)
    host_np = host.numpy()
    points_obb_batch(host_np, offsets)
    e2e_steps = max(3, min(a.steps, 10))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        points_obb_batch(host_np, offsets)
    e2e_s = time.perf_counter() - t0
    e2e_min = -dist.max(-(total * e2e_steps / e2e_s / 1e6))
    line = {
        "metric": "Batched DiTO-14 fit throughput (Mpoints/s)", "value": round(value, 3), "unit": "Mpoints/s",
        "n_gpus": dist.world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(total_ms / a.steps, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: anisotropic Gaussian clouds (sigma log-U[0.01,5] per axis), Haar rotation, "
                "U[-100,100]^3 offset; sizes log-U[64,262144]",
        "config": {"workload": "dito_batch", "sets_per_gpu": a.sets, "points_per_gpu": total, "point_bytes": 12,
                   "l2": f"{12 * total / 1e9:.2f} GB of points per step (> 126 MB L2), no flush",
                   "launch": "one graph: memset + one persistent kernel", "tuning": tuning,
                   "autotuned_ms": tuned_ms, "parallelism": f"replicas{dist.world}"},
        "kernels": kernel_table(prof, a.steps, batch_bytes, peak),
        "gpu_launches": sum(v[0] for v in prof.values()), "roofline": roof,
        "per_call": {"value": round(pc_value, 3), "unit": "Mpoints/s", "ms_per_batch": round(pc_ms, 3),
                     "api": "obvh_dito_fit_async per set (2 kernels per set, grid sized to the set's 2,048-point "
                            "tiles), same device buffer, the 4,096 calls replayed from one CUDA graph",
                     "speedup": round(value / pc_value, 2),
                     "host_loop_ms_per_batch": round(host_loop_ms, 3),
                     "host_loop_speedup": round(value / (total / (host_loop_ms / 1e3) / 1e6), 2)},
        "e2e": {"value": round(dist.world * e2e_min, 3), "unit": "Mpoints/s", "h2d_bytes_per_step": 12 * total,
                "d2h_bytes_per_step": 60 * a.sets + 4, "api": "obvh_points_obb_batch, pinned host"},
        "clocks": clocks,
    }
    if dist.rank == 0 and dist.world == 1:
        import oracle
        threads = os.cpu_count() or 1
        off = np.asarray(offsets, np.int64)
        oracle.ref_dito14_batch(host_np, off[:65], threads)
        t0 = time.perf_counter()
        oracle.ref_dito14_batch(host_np, off, threads)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": round(total / dt / 1e6, 3), "unit": "Mpoints/s", "cores": threads,
                                "kind": "reference",
                                "sample": f"the whole {a.sets}-set batch once ({dt:.1f} s), reference DiTO_14 "
                                          f"(oracle/_ref), one set per thread"}
    return line


def bench_batch_reference(a, dist):
    """The reference's CPU DiTO_14 over the batch, one set per host thread."""
    import numpy as np
    import oracle
    from obvh_b200 import workloads
    try:
        import torch
        dev = "cuda" if torch.cuda.is_available() else "cpu"
        pts, offsets = workloads.gaussian_sets_torch(a.sets, seed=3, device=dev)
        host = pts.cpu().numpy()
    except Exception:
        host, offsets = workloads.gaussian_sets(a.sets, seed=3)
    host = np.ascontiguousarray(host, dtype=np.float32)
    off = np.asarray(offsets, np.int64)
    total = int(off[-1])
    threads = os.cpu_count() or 1
    for _ in range(a.warmup):
        oracle.ref_dito14_batch(host, off[:65], threads)
    times = []
    for _ in range(a.steps):
        t0 = time.perf_counter()
        oracle.ref_dito14_batch(host, off, threads)
        times.append(time.perf_counter() - t0)
    value = total * len(times) / sum(times) / 1e6
    return {"metric": "Batched DiTO-14 fit throughput (Mpoints/s)", "impl": "reference", "value": round(value, 3),
            "unit": "Mpoints/s", "n_gpus": dist.world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": round(1e3 * sum(times) / len(times), 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (same generator as the ours arm)",
            "config": {"workload": "dito_batch", "sets_per_gpu": a.sets, "points_per_gpu": total},
            "cpu_baseline": {"value": round(value, 3), "unit": "Mpoints/s", "cores": threads, "kind": "reference",
                             "sample": f"the whole {a.sets}-set batch per step, one set per thread "
                                       f"(warm-up steps on the first 64 sets)"},
            "e2e": {"value": round(value, 3), "unit": "Mpoints/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def _mesh_batch_inputs(n_meshes, seed, dev):
    """Thin-triangle soups (the configs[1] generator) of log-uniform sizes
    64..16,384 triangles, packed: (verts, faces int32 [F, 4], vertex and face
    CSR offsets as numpy uint64)."""
    import numpy as np
    import torch
    from obvh_b200 import workloads
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(64), np.log(16384), size=n_meshes)).astype(np.int64)
    vs, fs = [], []
    for k, n in enumerate(sizes):
        v, f = workloads.triangle_soup_torch(int(n), seed=seed * 100003 + k, device=dev)
        vs.append(v)
        fs.append(f)
    vo = np.concatenate([[0], np.cumsum([v.shape[0] for v in vs])]).astype(np.uint64)
    fo = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    return torch.cat(vs).contiguous(), torch.cat(fs).contiguous(), vo, fo


def bench_mesh_batch_ours(a, dist):
    import numpy as np
    import torch
    from obvh_b200 import _native, bvh

    dev = torch.device("cuda", torch.cuda.current_device())
    verts, faces, vo, fo = _mesh_batch_inputs(a.meshes, 5 + dist.rank, dev)
    sizes = np.diff(fo).astype(np.int64)
    nodes = int(np.sum(2 * sizes - 1))
    batch = bvh.BuildBatch(vo, fo, flags=bvh.BUILD_OBBS | bvh.BUILD_COLLAPSE, device=dev)
    out = batch.outputs()
    stream = torch.cuda.current_stream(dev)
    batch.capture(verts, faces, out)
    sampler = ClockSampler(dev.index, enabled=not a.profile)
    total_ms, prof, clocks = timed_steps(a, dist, lambda j: batch.launch(stream), sampler, stream)
    err, slots = batch.status(stream)
    if err:
        raise RuntimeError(f"device error word {err}")
    if a.profile:
        return {"profile": "mesh_batch", "meshes": a.meshes, "ms_per_step": total_ms / a.steps, "kernels": prof}
    peak, peak_kind = peaks()
    ms_step = total_ms / a.steps
    value = dist.world * nodes / (ms_step / 1e3) / 1e6
    # the whole-build bytes of the tree workload, per mesh: 164 B per node + 52 B per triangle
    batch_bytes = {"mesh_batch_graph": int(np.sum(164 * (2 * sizes - 1) + 52 * sizes))}
    roof = roofline(prof, batch_bytes, peak, peak_kind)

    # plain per-call path: obvh_build_async per mesh on the same device buffers,
    # enqueued back to back on one stream (no waits between meshes)
    lib = _native.lib()
    nmax = int(sizes.max())
    ws = torch.empty(int(lib.obvh_build_workspace_bytes(nmax)), dtype=torch.uint8, device=dev)
    S = ctypes.c_void_p(stream.cuda_stream)
    _native.check(lib.obvh_build_workspace_init(ctypes.c_void_p(ws.data_ptr()), nmax, S))
    P = {k: t.data_ptr() for k, t in out.items()}
    vb, fb = verts.data_ptr(), faces.data_ptr()
    calls = []
    for m in range(a.meshes):
        nb, f0, n = batch.node_offset(m), int(fo[m]), int(sizes[m])
        calls.append([ctypes.c_void_p(vb + 12 * int(vo[m])), ctypes.c_void_p(fb + 16 * f0), n, 3,
                      ctypes.c_float(1.2), ctypes.c_float(1.0),
                      ctypes.c_void_p(P["nodes"] + 36 * nb), ctypes.c_void_p(P["parents"] + 4 * nb),
                      ctypes.c_void_p(P["counts"] + 4 * nb), ctypes.c_void_p(P["costs"] + 4 * nb),
                      ctypes.c_void_p(P["bounds"] + 48 * m), ctypes.c_void_p(P["obbs"] + 60 * nb),
                      ctypes.c_void_p(P["transforms"] + 64 * nb), ctypes.c_void_p(P["collapsed"] + 36 * nb),
                      ctypes.c_void_p(P["primitives"] + 4 * f0), ctypes.c_void_p(ws.data_ptr()), S])

    def per_call():
        for c in calls:
            e = lib.obvh_build_async(*c)
            if e:
                _native.check(e)
    per_call()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    per_call()
    e1.record(stream)
    torch.cuda.synchronize()
    pc_ms = e0.elapsed_time(e1)
    pc_value = -dist.max(-(nodes / (pc_ms / 1e3) / 1e6)) * dist.world

    # end to end: the packed meshes from pinned host memory every step, the
    # graph, the per-mesh slot counts read back (each step waited for)
    hv = torch.empty_like(verts, device="cpu").pin_memory()
    hf = torch.empty_like(faces, device="cpu").pin_memory()
    hv.copy_(verts)
    hf.copy_(faces)
    e2e_steps = max(3, min(a.steps, 10))

    def e2e_step():
        verts.copy_(hv, non_blocking=True)
        faces.copy_(hf, non_blocking=True)
        batch.launch(stream)
        batch.status(stream)
    e2e_step()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    serial_s = time.perf_counter() - t0

    # streamed: batch j+1's meshes are copied in on a second stream while
    # batch j builds (two input buffers, each with its own captured graph over
    # the same outputs); every step reads the meshes' boxes back
    verts2, faces2 = torch.empty_like(verts), torch.empty_like(faces)
    batch2 = bvh.BuildBatch(vo, fo, flags=bvh.BUILD_OBBS | bvh.BUILD_COLLAPSE, device=dev)
    batch2.capture(verts2, faces2, out)
    ins = [(verts, faces, batch), (verts2, faces2, batch2)]
    copy_stream = torch.cuda.Stream(dev)
    h2d_done = [torch.cuda.Event() for _ in range(2)]
    build_done = [torch.cuda.Event() for _ in range(2)]
    nbox = out["bounds"].numel()
    res = [torch.empty(nbox, dtype=out["bounds"].dtype, pin_memory=True) for _ in range(2)]

    def issue(j):
        v, f, b = ins[j & 1]
        with torch.cuda.stream(copy_stream):
            if j >= 2:
                copy_stream.wait_event(build_done[j & 1])
            v.copy_(hv, non_blocking=True)
            f.copy_(hf, non_blocking=True)
            h2d_done[j & 1].record(copy_stream)
        stream.wait_event(h2d_done[j & 1])
        b.launch(stream)
        build_done[j & 1].record(stream)
        res[j & 1].copy_(out["bounds"].view(-1), non_blocking=True)

    for j in range(2):
        issue(j)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for j in range(e2e_steps):
        issue(j)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    del batch2
    e2e_min = -dist.max(-(nodes * e2e_steps / e2e_s / 1e6))
    serial_min = -dist.max(-(nodes * e2e_steps / serial_s / 1e6))
    info = batch.info()
    line = {
        "metric": "Batched LBVH + OBB-tree + collapse builds (Mnodes/s)", "value": round(value, 3),
        "unit": "Mnodes/s", "n_gpus": dist.world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": round(ms_step, 5), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic: thin random triangle soups (configs[1] generator), sizes log-U[64,16384], seeded",
        "config": {"workload": "mesh_batch", "meshes_per_gpu": a.meshes, "triangles_per_gpu": int(sizes.sum()),
                   "nodes_per_gpu": nodes, "launch": "one graph: memset + one persistent kernel, one mesh per CTA",
                   "plan": info, "l2": f"{(12 * int(vo[-1]) + 16 * int(fo[-1])) / 1e6:.0f} MB of meshes in, "
                                       "~1.5 GB written per step, no flush",
                   "parallelism": f"replicas{dist.world}"},
        "kernels": kernel_table(prof, a.steps, batch_bytes, peak),
        "gpu_launches": sum(v[0] for v in prof.values()), "roofline": roof,
        "per_call": {"value": round(pc_value, 3), "unit": "Mnodes/s", "ms_per_batch": round(pc_ms, 3),
                     "api": "obvh_build_async per mesh (the whole-GPU chain), back to back on one stream",
                     "speedup": round(value / pc_value, 2)},
        "e2e": {"value": round(dist.world * e2e_min, 3), "unit": "Mnodes/s",
                "h2d_bytes_per_step": int(verts.numel() * 4 + faces.numel() * 4),
                "d2h_bytes_per_step": int(nbox * 4),
                "api": "obvh_build_batch_launch from pinned host meshes; the copy of batch j+1 (second stream) "
                       "overlaps the build of batch j; the meshes' boxes read back every step",
                "serial": {"value": round(dist.world * serial_min, 3),
                           "api": "the same calls with each step's copy, build and status read waited for in turn"}},
        "clocks": clocks,
    }
    if dist.rank == 0 and dist.world == 1:
        line["cpu_baseline"] = cpu_mesh_batch_baseline(verts, faces, vo, fo)
    return line


def cpu_mesh_batch_baseline(verts, faces, vo, fo, budget_s=8.0):
    """The oracle port of the same builds on one host core, over the batch's
    first meshes until the time budget is spent."""
    from oracle import bvh as ref
    hv, hf = verts.cpu().numpy(), faces.cpu().numpy().view("uint32")
    done_nodes, m, t0 = 0, 0, time.perf_counter()
    while m < len(fo) - 1 and time.perf_counter() - t0 < budget_s:
        v = hv[int(vo[m]):int(vo[m + 1])]
        f = hf[int(fo[m]):int(fo[m + 1])]
        r = ref.lbvh_build(v, f)
        ref.obb_tree(r["nodes"], r["parents"], v, f)
        ref.collapse(r["nodes"], r["parents"], r["counts"], r["costs"])
        done_nodes += 2 * f.shape[0] - 1
        m += 1
    dt = time.perf_counter() - t0
    return {"value": round(done_nodes / dt / 1e6, 4), "unit": "Mnodes/s", "cores": 1, "kind": "port",
            "sample": f"the first {m} meshes of the batch ({dt:.1f} s), oracle C restatement"}


def bench_mesh_batch_reference(a, dist):
    """The oracle port of the batch's builds on this host's cores: each step,
    every host thread builds one sample of the batch's meshes (the first 64,
    about a tenth of a second of work per thread)."""
    import numpy as np
    import torch
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    verts, faces, vo, fo = _mesh_batch_inputs(a.meshes, 5, dev)
    hv, hf = verts.cpu().numpy(), faces.cpu().numpy().view(np.uint32)
    sample = min(64, len(fo) - 1)
    nodes = int(sum(2 * (int(fo[m + 1]) - int(fo[m])) - 1 for m in range(sample)))
    from oracle import bvh as ref

    def work():
        for m in range(sample):
            v = hv[int(vo[m]):int(vo[m + 1])]
            f = hf[int(fo[m]):int(fo[m + 1])]
            r = ref.lbvh_build(v, f)
            ref.obb_tree(r["nodes"], r["parents"], v, f)
            ref.collapse(r["nodes"], r["parents"], r["counts"], r["costs"])
    threads = host_threads()
    times = parallel_steps(a, work, threads)
    value = threads * nodes * len(times) / sum(times) / 1e6
    return {"metric": "Batched LBVH + OBB-tree + collapse builds (Mnodes/s)", "impl": "reference",
            "value": round(value, 4), "unit": "Mnodes/s", "n_gpus": dist.world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(1e3 * sum(times) / len(times), 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (same generator as the ours arm)",
            "config": {"workload": "mesh_batch", "meshes_per_gpu": a.meshes, "sample_meshes": sample},
            "cpu_baseline": {"value": round(value, 4), "unit": "Mnodes/s", "cores": threads, "kind": "port",
                             "sample": f"{threads} threads each building the batch's first {sample} meshes per "
                                       "step, oracle C restatement"},
            "e2e": {"value": round(value, 4), "unit": "Mnodes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def _serve_requests(n_req, seed, dev):
    """The served mix: 70% DiTO fits of Gaussian clouds (1k..4M points,
    log-uniform), 30% LBVH + OBB-tree + collapse builds of thin-triangle
    soups (10k..2M triangles, log-uniform); inputs resident on the device."""
    import math
    import numpy as np
    from obvh_b200 import workloads
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(n_req):
        if rng.uniform() < 0.7:
            n = int(math.exp(rng.uniform(math.log(1e3), math.log(4e6))))
            reqs.append(("fit", workloads.gaussian_cloud_torch(n, rng, device=dev), n))
        else:
            n = int(math.exp(rng.uniform(math.log(1e4), math.log(2e6))))
            v, f = workloads.triangle_soup_torch(n, seed=int(rng.integers(0, 2 ** 31)), device=dev)
            reqs.append(("build", (v, f), n))
    return reqs


def bench_serve_ours(a, dist):
    import threading
    import numpy as np
    import torch
    from obvh_b200 import _native, bvh
    from obvh_b200.server import Server

    dev = torch.device("cuda", torch.cuda.current_device())
    lib = _native.lib()
    reqs = _serve_requests(a.requests, 4 + dist.rank, dev)
    torch.cuda.synchronize()
    n_fit = sum(1 for r in reqs if r[0] == "fit")
    pts = sum(r[2] for r in reqs if r[0] == "fit")
    nodes = sum(2 * r[2] - 1 for r in reqs if r[0] == "build")
    stream = torch.cuda.current_stream(dev)
    S = ctypes.c_void_p(stream.cuda_stream)

    # serial plain per-call: one request at a time through the plain paths, each
    # call waited for before the next (the reference's kr_cuda_points_obb /
    # commit are blocking calls); inputs already on the device
    ws_fit = torch.zeros(int(lib.obvh_dito_workspace_bytes()), dtype=torch.uint8, device=dev)
    _native.check(lib.obvh_dito_workspace_init(ctypes.c_void_p(ws_fit.data_ptr()), S))
    nmax = max([r[2] for r in reqs if r[0] == "build"] or [1])
    builder = bvh.ObvhBuilder(dev)
    outs = builder.outputs(nmax)
    obb = torch.empty(15, dtype=torch.float32, device=dev)

    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    device_ms = {"fit": 0.0, "build": 0.0}

    def plain(r):
        ev[0].record(stream)
        if r[0] == "fit":
            p = r[1]
            _native.check(lib.obvh_dito_fit_async(ctypes.c_void_p(p.data_ptr()), r[2], 0, ctypes.c_void_p(obb.data_ptr()),
                                                  ctypes.c_void_p(ws_fit.data_ptr()), S))
        else:
            v, f = r[1]
            builder.build(bvh.Mesh.from_device(v, f), flags=3, ci=1.2, ct=1.0, stream=stream, out=outs)
        ev[1].record(stream)
        stream.synchronize()
        device_ms[r[0]] += ev[0].elapsed_time(ev[1])

    for r in reqs:  # warm-up over the whole list: workspaces sized, every kernel loaded
        plain(r)
    device_ms = {"fit": 0.0, "build": 0.0}
    t0 = time.perf_counter()
    for r in reqs:
        plain(r)
    serial_s = time.perf_counter() - t0
    serial_rps = len(reqs) / serial_s
    del outs
    torch.cuda.empty_cache()

    free, _ = torch.cuda.mem_get_info(dev)
    budget = int(min(120 << 30, free - (4 << 30)))

    def run(rate, host=None):
        """Submits every request (Poisson arrivals at `rate` req/s, or all at
        once for rate None), releases results in order; returns stats."""
        srv = Server(budget_bytes=budget, build_lanes=4)
        ids = [None] * len(reqs)
        ready = threading.Semaphore(0)

        def producer():
            rng = np.random.default_rng(99)
            t_next = time.perf_counter()
            for k, r in enumerate(reqs):
                if rate:
                    t_next += rng.exponential(1.0 / rate)
                    delay = t_next - time.perf_counter()
                    if delay > 0:
                        time.sleep(delay)
                if r[0] == "fit":
                    ids[k] = srv.submit_fit(host[k] if host else r[1])
                else:
                    ids[k] = srv.submit_build(*(host[k] if host else r[1]), flags=3, ci=1.2, ct=1.0)
                ready.release()

        t = threading.Thread(target=producer)
        t0 = time.perf_counter()
        t.start()
        for k in range(len(reqs)):
            ready.acquire()
            srv.wait(ids[k], 600_000)
            srv.release(ids[k])
        t.join()
        wall = time.perf_counter() - t0
        st = srv.stats()
        srv.close()
        return st, wall

    run(None)  # warm-up (plans, arena)
    # saturated: three runs without per-launch events (the serial comparator
    # has none either), the median reported; the kernel list comes from a
    # fourth run with an event pair around every launch
    sats = sorted((run(None)[0] for _ in range(3)), key=lambda st: st["span_s"])
    sat = sats[1]
    profile_enable(True)
    prof_st, _ = run(None)
    prof = profile_summary()
    profile_enable(False)
    served_rps = len(reqs) / sat["span_s"]
    sweep = {}
    for frac in (0.5, 1.0, 2.0, 4.0):
        rate = frac * serial_rps
        st, wall = run(rate)
        sweep[f"{frac:g}x_serial_rate"] = {"offered_rps": round(rate, 2), "served_rps": round(len(reqs) / wall, 2),
                                           "p50_ms": round(st["p50_ms"], 3), "p99_ms": round(st["p99_ms"], 3),
                                           "max_ms": round(st["max_ms"], 3), "fit_batches": st["fit_batches"]}
    # end to end: the same mix from pinned host memory, copied in by the server
    host = []
    for r in reqs:
        if r[0] == "fit":
            host.append(r[1].cpu().pin_memory().numpy())
        else:
            host.append((r[1][0].cpu().pin_memory().numpy(), r[1][1].cpu().pin_memory().numpy().view(np.uint32)))
    e2e, e2e_wall = run(None, host)
    h2d = sum(12 * r[2] if r[0] == "fit" else 12 * 3 * r[2] + 16 * r[2] for r in reqs)
    return {
        "metric": "Served mixed requests throughput (requests/s)", "value": round(served_rps, 3), "unit": "requests/s",
        "n_gpus": dist.world, "steps": 1, "warmup": 1, "ms_per_step": round(1e3 * sat["span_s"], 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: 70% Gaussian-cloud fits (1k..4M points), 30% thin-triangle soup builds (10k..2M), "
                "log-uniform sizes, seeded",
        "config": {"workload": "serve_mixed", "requests": len(reqs), "fits": n_fit, "builds": len(reqs) - n_fit,
                   "points": pts, "build_nodes": nodes, "hbm_budget_bytes": budget, "build_lanes": 4,
                   "inputs": "device-resident", "l2": "GBs of inputs per run (> 126 MB L2)",
                   "parallelism": f"replicas{dist.world}"},
        "served": {"runs_rps": [round(len(reqs) / st["span_s"], 3) for st in sats], "reported": "median of 3",
                   "profiled_run_rps": round(len(reqs) / prof_st["span_s"], 3),
                   "p50_ms": round(sat["p50_ms"], 3), "p99_ms": round(sat["p99_ms"], 3),
                   "fit_batches": sat["fit_batches"], "peak_arena_bytes": sat["peak_bytes"],
                   "mpoints_per_s": round(pts / sat["span_s"] / 1e6, 2),
                   "mnodes_per_s": round(nodes / sat["span_s"] / 1e6, 2)},
        "per_call": {"value": round(serial_rps, 3), "unit": "requests/s", "seconds": round(serial_s, 4),
                     "api": "obvh_dito_fit_async / obvh_build_async, one request at a time, each waited for",
                     "speedup": round(served_rps / serial_rps, 2),
                     "lone_device_ms": {k: round(x, 3) for k, x in device_ms.items()},
                     "lone_device_note": "each request's own device time in the serial loop (CUDA events around "
                                         "its kernels, GPU otherwise idle), summed"},
        "poisson_sweep": sweep,
        "kernels": {k: {"launches": v[0], "ms": round(v[1], 4)} for k, v in prof.items()},
        "gpu_launches": sum(v[0] for v in prof.values()),
        "gpu_launches_note": "counted in the profiled run; each timed run launches the same kernels",
        "roofline": None,
        "e2e": {"value": round(len(reqs) / e2e["span_s"], 3), "unit": "requests/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": 60 * n_fit, "api": "obvh_server_submit_fit / _build from pinned host memory",
                "p50_ms": round(e2e["p50_ms"], 3), "p99_ms": round(e2e["p99_ms"], 3)},
    }


def extra_workloads(a, dist, line):
    """The default line at 1 GPU also carries the other measured workloads
    (the 100M-point DiTO fit, the 4,096-set batch, the served mix), each with
    its own CUDA-event timing, clocks, roofline, per-call comparison and e2e,
    so that every target is timed in the same run.  About a minute extra."""
    import copy
    import gc
    import torch
    subs = {"dito_100M": ("dito", 20, 5, bench_dito_ours), "dito_batch": ("dito_batch", 10, 3, bench_batch_ours),
            "serve": ("serve", 1, 1, bench_serve_ours)}
    for key, (workload, steps, warmup, fn) in subs.items():
        b = copy.copy(a)
        b.workload, b.steps, b.warmup = workload, steps, warmup
        if workload == "serve":
            b.requests = 200
        t0 = time.perf_counter()
        sub = fn(b, dist)
        sub.pop("kernels", None)
        sub["wall_s"] = round(time.perf_counter() - t0, 1)
        line[key] = sub
        gc.collect()
        torch.cuda.empty_cache()
    # What any schedule of the served mix needs at least: its build nodes at
    # the 2M-triangle build's own rate (this line's value, a build that fills
    # the GPU alone) plus its fit points at 24 B/point at the HBM peak; the
    # serial per-call time over that bounds the served speed-up on this mix.
    sv = line["serve"]
    peak, peak_kind = peaks()
    floor_s = (sv["config"]["build_nodes"] / (line["value"] * 1e6 / dist.world)
               + 24 * sv["config"]["points"] / (peak * 1e9))
    pc = sv["per_call"]
    pc["speedup_bound"] = round(pc["seconds"] / floor_s, 2)
    pc["bound_note"] = ("serial per-call seconds over (build nodes at this line's 2M-triangle build rate + fit points "
                        f"at 24 B/point at the {peak_kind} HBM peak): the mix is build-bound")
    d = line["dito_100M"]
    # the whole fit against 24 B/point (two compulsory passes over 12-byte points)
    fit_gbs = 24 * d["config"]["points_per_gpu"] / (d["ms_per_step"] / 1e3) / 1e9
    d["fit_roofline"] = {"bound": "hbm", "achieved": round(fit_gbs, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(fit_gbs / peak, 4), "bytes_per_point": 24,
                         "note": f"both passes, one fit per step, peak {peak_kind}"}


def main():
    a = parse_args()
    dist = Dist()
    if a.impl == "reference":
        if dist.world > 1 and dist.rank != 0:
            return
        if a.workload in ("dito", "dito_batch"):
            import oracle
            if not oracle.ref_available():
                print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_dito.so was not built"}))
                return
            ref = bench_dito_reference if a.workload == "dito" else bench_batch_reference
            print(json.dumps(ref(a, dist)), flush=True)
        elif a.workload == "atrbvh_obb_tree":
            print(json.dumps(bench_atrbvh_reference(a, dist)), flush=True)
        elif a.workload == "obvh_pack":
            print(json.dumps(bench_pack_reference(a, dist)), flush=True)
        elif a.workload == "obvh_trace":
            print(json.dumps(bench_trace_reference(a, dist)), flush=True)
        elif a.workload == "mesh_batch":
            print(json.dumps(bench_mesh_batch_reference(a, dist)), flush=True)
        elif a.workload == "obvh_trace_compressed":
            print(json.dumps({"impl": "reference", "unavailable": "the reference's compressed traversal exists only "
                              "as a GPU kernel (pinned against this build in the GPU tests); there is no CPU form"}))
        else:
            print(json.dumps(bench_tree_reference(a, dist)), flush=True)
        return
    dist.init()
    try:
        run = {"lbvh_obb_tree": bench_tree_ours, "atrbvh_obb_tree": lambda a, d: bench_tree_ours(a, d, atrbvh=True),
               "dito": bench_dito_ours, "dito_batch": bench_batch_ours, "serve": bench_serve_ours,
               "obvh_pack": bench_pack_ours, "obvh_trace": bench_trace_ours,
               "obvh_trace_compressed": bench_trace_compressed_ours, "mesh_batch": bench_mesh_batch_ours}
        line = run[a.workload](a, dist)
        if a.workload == "lbvh_obb_tree" and dist.world == 1 and not (a.profile or a.no_extras):
            extra_workloads(a, dist, line)
        if dist.rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
