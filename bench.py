"""Benchmark of the ray-element hot path: batched point location.

Workload (one step): locate 16,777,216 query points (uniform in a cube
padded so ~8% lie outside the mesh) in a 64^3 order-2 Bernstein hex mesh
whose elements are trilinear maps of a randomly displaced vertex lattice
(15% of the element size), Newton tolerance 1e-5 in reference space,
at most 20 steps.  Mesh, BVH and queries are built once before timing; the
timed step is the hot path (query ordering + traversal + Newton).

Arms
  ours (default)      the batched path: learned initial guess when a trained
                      guess model is present, Morton-ordered queries,
                      persistent work-queue kernel with an autotuned shape
  --impl reference    the reference's own CPU implementation (Devil Ray
                      compiled from its sources, OpenMP, all host threads)
                      on a bounded sample of the same workload

Timing: W warm-up steps, then K steps between CUDA events on the launching
stream with a device synchronize on both sides; under torchrun every rank
locates its own 16M queries (weak scaling) and the slowest rank's time
counts.  The working set (201 MB of queries, 553 MB of BVH nodes) is larger
than the 126 MB L2.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = "locate_64"
N_QUERIES = 16_777_216
TOL = 1e-5
MAX_STEPS = 20
METRIC = "located pts/s (Newton-resolved, tol 1e-5)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--queries", type=int, default=N_QUERIES)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample", type=int, default=0,
                    help="reference CPU sample size (0 = sized for ~15 s)")
    ap.add_argument("--profile", action="store_true",
                    help="profiling run: fixed launch shape, only the timed steps "
                         "(no tuning, plain/e2e/statistics/CPU legs)")
    return ap.parse_args()


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def reference_arm(args, rank, world):
    """--impl reference: the reference's CPU Mesh::locate (oracle/_ref)."""
    if rank != 0:
        return 0
    from devil_ray_b200 import meshgen
    from oracle import refpy
    if not refpy.available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/libdray_ref.so was not built"}))
        return 0
    m = meshgen.workload_mesh(WORKLOAD)
    r = refpy.RefHexMesh(m.order, m.ctrl_idx, m.xyz, m.field)
    t0 = time.perf_counter()
    r.bvh()
    build_s = time.perf_counter() - t0
    threads = refpy.num_threads()
    sample = args.cpu_sample or 131072
    q = meshgen.uniform_queries(args.queries, 1000 + rank)[:sample]
    for _ in range(max(args.warmup, 0) and 1):
        r.locate(q[:4096])
    times, located = [], 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        cell, _ = r.locate(q)
        times.append(time.perf_counter() - t0)
        located = int((cell >= 0).sum())
    t = float(np.mean(times))
    value = located / t
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "points/s",
            "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": WORKLOAD + " (reference CPU, sample per step)",
                       "queries_per_step": sample, "tol": 1e-4, "max_steps": 20,
                       "note": "reference Newton tolerance is hard-coded to 1e-4"},
            "cpu_baseline": {"value": value, "unit": "points/s", "cores": threads,
                             "kind": "reference",
                             "sample": f"{sample} of the 16M queries per step, BVH built once "
                                       f"({build_s:.1f} s, not timed)"},
            "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def cpu_baseline(mesh_data, queries, bvh_np):
    """Reference CPU locate on a bounded sample (about 10-20 s of work)."""
    from oracle import refpy
    if not refpy.available():
        return None
    r = refpy.RefHexMesh(mesh_data.order, mesh_data.ctrl_idx, mesh_data.xyz)
    t0 = time.perf_counter()
    r.bvh()
    build_s = time.perf_counter() - t0
    q = queries[:8192]
    t0 = time.perf_counter()
    r.locate(q)
    t_probe = time.perf_counter() - t0
    sample = int(min(len(queries), max(8192, 8192 * 12.0 / max(t_probe, 1e-3))))
    q = queries[:sample]
    t0 = time.perf_counter()
    cell, _ = r.locate(q)
    t = time.perf_counter() - t0
    located = int((cell >= 0).sum())
    return {"value": located / t, "unit": "points/s", "cores": refpy.num_threads(),
            "kind": "reference",
            "sample": f"{sample} of the 16M queries (reference tol 1e-4, 20 steps), "
                      f"{t:.1f} s; reference BVH build {build_s:.1f} s not timed"}


def main():
    args = parse()
    rank, world, local = dist_info()
    if args.impl == "reference":
        return reference_arm(args, rank, world)

    import torch
    from devil_ray_b200 import _lib as L
    from devil_ray_b200 import api, meshgen

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
        pg = dist

    m = meshgen.workload_mesh(WORKLOAD)
    queries = meshgen.uniform_queries(args.queries, 1000 + rank)
    mesh = api.UnstructuredMesh(m.ctrl_idx, m.xyz, m.order, device=dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    bvh = mesh.get_bvh()
    torch.cuda.synchronize()
    bvh_build_ms = 1e3 * (time.perf_counter() - t0)
    # BVH build timed again warm (first call includes lazy module loading)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    mesh.build_bvh()
    ev1.record()
    torch.cuda.synchronize()
    bvh_build_ms = ev0.elapsed_time(ev1)

    pts = torch.as_tensor(queries, device=dev)
    n = pts.shape[0]
    loc = api.BatchedLocator(mesh, tol=TOL, max_steps=MAX_STEPS, guess_mode=L.GUESS_ELEM_CENTER)
    if args.profile:
        best_cfg = L.DrbLocateConfig(128, 4, 64, 1)
        loc.config, tune_ms = best_cfg, 0.0
    else:
        best_cfg, tune_ms = loc.tune(pts[: min(n, 1 << 21)])
    cell = torch.empty(n, dtype=torch.int32, device=dev)
    ref = torch.empty((n, 3), dtype=torch.float32, device=dev)

    def step():
        loc.locate(pts, out=(cell, ref))

    # plain path (the reference's launch pattern on the GPU) for comparison
    def plain_step():
        mesh.locate(pts, tol=TOL, max_steps=MAX_STEPS, guess_mode=L.GUESS_ELEM_CENTER)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()

    def timed(fn, k):
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        for _ in range(k):
            fn()
        s1.record()
        torch.cuda.synchronize()
        ms = s0.elapsed_time(s1)
        if pg:
            t = torch.tensor([ms], device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    clocks = ClockSampler(local)
    clocks.start()
    launches0 = L.lib().drb_kernel_launches()
    total_ms = timed(step, args.steps)
    launches = L.lib().drb_kernel_launches() - launches0
    clk = clocks.stop()
    ms_step = total_ms / args.steps
    located = int((cell >= 0).sum().item())
    if args.profile:
        if rank == 0:
            print(json.dumps({"profile": True, "ms_per_step": ms_step, "queries": n,
                              "located": located, "launches_per_step": launches / args.steps}))
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return 0
    # statistics of the same queries (untimed): iterations, candidates, nodes
    _, _, it, ca, nd = loc.locate(pts, stats=True)
    mean_it = float(it.float().mean())
    mean_ca = float(ca.float().mean())
    mean_nd = float(nd.float().mean())
    hist = torch.bincount(it.long().clamp(max=40), minlength=41).cpu().numpy().tolist()
    # plain path
    for _ in range(2):
        plain_step()
    plain_ms = timed(plain_step, max(2, args.steps // 2)) / max(2, args.steps // 2)

    # persistent kernel alone (roofline): time it separately on a fixed order
    order = loc.order(pts)
    kern_ms = timed(lambda: loc.locate(pts, order=order, out=(cell, ref)), args.steps) / args.steps

    value = world * located / (ms_step * 1e-3)

    # algorithmic bytes per query (SURVEY 8d formula): point 12 B + Location
    # 16 B + per candidate one element's control points (nd x 12 B packed)
    # and reference box 24 B + 64 B per inner node visited
    nd_dofs = (m.order + 1) ** 3
    bytes_q = 12 + 16 + mean_ca * (nd_dofs * 12 + 24) + 64 * mean_nd
    achieved_gbs = n * bytes_q / (kern_ms * 1e-3) / 1e9
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)

    # end to end through the public API: pinned host queries -> device ->
    # batched locate -> Location records back to pinned host memory
    host_pts = torch.from_numpy(queries).pin_memory()
    host_cell = torch.empty(n, dtype=torch.int32).pin_memory()
    host_ref = torch.empty((n, 3), dtype=torch.float32).pin_memory()
    dpts = torch.empty_like(pts)

    def e2e_step():
        dpts.copy_(host_pts, non_blocking=True)
        loc.locate(dpts, out=(cell, ref))
        host_cell.copy_(cell, non_blocking=True)
        host_ref.copy_(ref, non_blocking=True)

    e2e_step()
    e2e_ms = timed(e2e_step, args.steps) / args.steps
    e2e_located = int((host_cell >= 0).sum())
    e2e_value = world * e2e_located / (e2e_ms * 1e-3)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(m, queries, None)
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"error": str(exc)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": "locate_64: 64^3 hex order 2, trilinear distortion 15%, "
                                   "16M uniform queries (8% outside), tol 1e-5, 20 steps",
                       "queries_per_gpu": n, "elements": m.n_elem, "bvh_leaves": bvh.n_leaf,
                       "guess": "element centre", "launch_config": best_cfg.as_dict(),
                       "l2": "inputs larger than L2 (201 MB queries, 553 MB BVH nodes)",
                       "parallelism": f"replicas x{world}, queries sharded, no collective"},
            "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": peak, "unit": "GB/s",
                         "frac": achieved_gbs / peak, "traffic": None,
                         "kernel": "locate_persistent_kernel",
                         "bytes_per_query": bytes_q, "kernel_ms": kern_ms},
            "e2e": {"value": e2e_value, "unit": "points/s",
                    "h2d_bytes_per_step": int(n * 12), "d2h_bytes_per_step": int(n * 16),
                    "ms_per_step": e2e_ms},
            "gpu_launches": int(launches),
            "clocks": clk,
            "stats": {"located_fraction": located / n, "mean_newton_iters": mean_it,
                      "mean_candidates": mean_ca, "mean_nodes_visited": mean_nd,
                      "iteration_histogram": hist},
            "plain": {"ms_per_step": plain_ms, "value": world * located / (plain_ms * 1e-3),
                      "note": "one thread per query in input order (reference launch pattern)"},
            "bvh_build_ms": bvh_build_ms, "tune_ms": tune_ms,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
