"""Benchmark of the B200 spectral path-tracing backend.

`python bench.py --gpus N --steps K --warmup W` prints one JSON line (rank 0).

Workloads (all inputs synthetic and seeded, FP32):
  raycast  8,388,608-triangle soup (centroids U[0,1]^3, edges N(0, 0.002^2)) and
           16,777,216 incoherent rays (origins U[-0.1,1.1]^3, directions uniform on the
           sphere, tmax inf); one step = one closest-hit batch over all rays.
           Inputs (768 MB of rays + ~1 GB of BVH) exceed the 126 MB L2, so no flush
           is needed between steps.
`--impl reference` times the CPU path on the host cores (rank 0 only) on the same
workload: the CPU oracle's closest-hit traversal over a bounded sample of the rays.
Multi-GPU: one process per GPU, each rank traces its own ray batch (different seed)
against its own copy of the scene; no collective on the data path ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "filianore-core_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

N_TRI = 1 << 23
N_RAYS = 1 << 24
NODE_BYTES = 80
TRI_BYTES = 48
RAY_BYTES = 32
HIT_BYTES = 16


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": d["hbm_gbs"], "src": "measured"}
    return {"hbm_gbs": 6650.0, "src": "fallback"}


class ClockSampler:
    """nvidia-smi sampling during the timed region (clock, power, throttle reasons)."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"fl_clocks_{os.getpid()}.csv")

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, name in enumerate(names):
                if r[5 + k].strip() == "Active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": sorted(reasons),
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows)}


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def raycast_workload(rank):
    from filianore_b200 import scenes
    tris = scenes.triangle_soup(N_TRI, seed=1)
    org, dirs = scenes.incoherent_rays(N_RAYS, seed=2 + rank)
    return tris, org, dirs


def cpu_reference(args, world, rank):
    """CPU baseline on the host cores: the oracle's BVH closest-hit over a ray sample."""
    if rank != 0:
        return None
    import oracle
    tris, org, dirs = raycast_workload(0)
    t0 = time.perf_counter()
    bvh = oracle.CpuBVH(tris)
    build_s = time.perf_counter() - t0
    cores = os.cpu_count() or 1
    sample = 1 << 20
    times = []
    for i in range(args.warmup + args.steps):
        sl = slice((i * sample) % N_RAYS, (i * sample) % N_RAYS + sample)
        t0 = time.perf_counter()
        bvh.trace(org[sl], dirs[sl], nthreads=cores)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    mrays = sample / statistics.mean(times) / 1e6
    return {"value": round(mrays, 3), "unit": "Mrays/s", "cores": cores, "kind": "port",
            "sample": f"{sample} of the {N_RAYS} incoherent rays per step against the full {N_TRI}-triangle soup "
                      f"(oracle binned-SAH BVH, build {build_s:.1f} s not timed)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    world, rank, local = dist_setup(args.gpus)
    config = {"workload": "raycast: 8,388,608-triangle soup, 16,777,216 incoherent rays, closest hit",
              "n_tri": N_TRI, "rays_per_gpu": N_RAYS, "l2": "inputs larger than L2 (no flush)",
              "parallelism": f"replicas x{world}"}

    if args.impl == "reference":
        if rank == 0:
            cb = cpu_reference(args, world, rank)
            line = {"metric": "Mrays/s", "value": cb["value"], "unit": "Mrays/s", "n_gpus": world,
                    "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                    "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config,
                    "impl": "reference", "cpu_baseline": cb,
                    "e2e": {"value": cb["value"], "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                            "d2h_bytes_per_step": 0}}
            print(json.dumps(line), flush=True)
        return

    import torch
    import filianore_b200 as fb
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    tris, org, dirs = raycast_workload(rank)
    from filianore_b200 import scenes
    sc = scenes.Scene(tris, np.zeros(N_TRI, np.uint32), [{"type": 0, "rgb": (0.5, 0.5, 0.5)}], [], None)
    ctx = fb.Context(local)
    scene = ctx.scene(sc)
    info = scene.info()
    d_org = torch.from_numpy(org).cuda()
    d_dir = torch.from_numpy(dirs).cuda()
    d_hits = torch.empty((N_RAYS, 4), dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    nodes, trisv = scene.trace_count(d_org, d_dir)
    alg_bytes = N_RAYS * (RAY_BYTES + HIT_BYTES) + NODE_BYTES * nodes + TRI_BYTES * trisv

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        scene.trace_closest(d_org, d_dir, out=d_hits, stream=stream)
    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record()
    for k in range(args.steps):
        ev[k][0].record()
        scene.trace_closest(d_org, d_dir, out=d_hits, stream=stream)
        ev[k][1].record()
    t_end.record()
    barrier()
    clk = clocks.stop()
    total_ms = t_start.elapsed_time(t_end)
    per_launch = [a.elapsed_time(b) for a, b in ev]
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = world * N_RAYS * args.steps / (total_ms / 1e3) / 1e6

    # end to end through the C ABI with pinned host buffers (H2D rays, D2H hits inside the call)
    h_org = torch.from_numpy(org).pin_memory()
    h_dir = torch.from_numpy(dirs).pin_memory()
    h_hits = torch.empty((N_RAYS, 4), dtype=torch.int32).pin_memory()
    import ctypes as C
    L = fb.lib()
    e2e_steps = max(2, args.steps // 2)
    L.fl_trace_closest(scene.h, C.c_void_p(h_org.data_ptr()), C.c_void_p(h_dir.data_ptr()), N_RAYS,
                       C.c_void_p(h_hits.data_ptr()), fb.FL_MEM_HOST, None)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        fb.check(L.fl_trace_closest(scene.h, C.c_void_p(h_org.data_ptr()), C.c_void_p(h_dir.data_ptr()), N_RAYS,
                                    C.c_void_p(h_hits.data_ptr()), fb.FL_MEM_HOST, None), ctx.h)
    barrier()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": round(world * N_RAYS / e2e_s / 1e6, 3), "unit": "Mrays/s",
           "h2d_bytes_per_step": N_RAYS * RAY_BYTES, "d2h_bytes_per_step": N_RAYS * HIT_BYTES}

    peaks = load_peaks()
    launch_ms = statistics.mean(per_launch)
    achieved = alg_bytes / (launch_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": None,
                "peak_src": peaks["src"], "kernel": "k_trace<closest>",
                "alg_bytes_per_launch": int(alg_bytes), "nodes_per_ray": round(nodes / N_RAYS, 2),
                "tris_per_ray": round(trisv / N_RAYS, 2)}
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_reference(args, 1, 0)
    if rank == 0:
        line = {"metric": "Mrays/s", "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": config, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": args.steps, "clocks": clk,
                "bvh": {"nodes": info["n_nodes"], "depth": info["max_depth"], "build_ms": round(info["build_ms"], 2),
                        "bytes": info["bvh_bytes"]}}
        print(json.dumps(line), flush=True)
    scene.close()
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
