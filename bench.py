"""Benchmark of the B200 spectral path-tracing backend.

`python bench.py --gpus N --steps K --warmup W` prints one JSON line (rank 0).

Workloads (all inputs synthetic and seeded, FP32 geometry):
  render (default)  procedural scene of 1,048,578 triangles: 64 UV spheres of 16,384
           triangles (radial value-noise displacement, amplitude 0.05 r) on a 2-triangle
           ground plane; 40% Lambert, 40% GGX conductor (eta 0.2, k 3.9), 20% rough
           dielectric (IOR 1.5); constant environment 0.5 plus one sphere light;
           1920x1080, 64 spp, max depth 16, 4 hero wavelengths. One step = one frame.
           The working set (path state ~0.8 GB per wave, BVH ~60 MB, film 50 MB) is
           larger than the 126 MB L2, so no flush is needed between steps.
           The render line also carries a "raycast" object: the ray-cast workload below,
           measured in the same run (both ray sets, roofline, end to end).
  raycast  8,388,608-triangle soup (centroids U[0,1]^3, edges N(0, 0.002^2)) and two ray
           sets: 16,777,216 incoherent rays (origins U[-0.1,1.1]^3, directions uniform on
           the sphere, tmax inf) and 4096 x 4096 pinhole primary rays towards the cube's
           centre; one step = one closest-hit batch. Inputs exceed L2.
`--impl reference` times the CPU implementation of the same workload on the host cores
(rank 0 only): the CPU oracle, a restatement of the reference's integrator pinned
bit-exact against the reference's own build, on a bounded sample of pixels or rays.
Multi-GPU: one process per GPU. render: each rank renders its own 64-spp pass of the
same image (samples offset by rank) and the FP64 films are summed to rank 0 with one
NCCL reduce per frame; raycast: each rank traces its own ray batch (no collective).
Per-GPU work is fixed as N grows ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import ctypes as C
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
RENDER = {"width": 1920, "height": 1080, "spp": 64, "depth": 16}
# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of the roofline kernels,
# measured with one-pass ncu captures of this command on a B200:
#   raycast: one k_trace launch over the full 16,777,216 rays: 32.73 + 1.21 GB
#   render:  k_trace_paths + k_trace_rays2 over the first 8 of the frame's 64 waves
#            (272 launches): 5.762 + 0.368 GB, times 8 for the frame
# DRAM bytes (read + write) of the roofline kernels from ncu captures of this code: the
# render's traversal kernels over one whole timed frame (48 streaming iterations), and one
# k_trace launch of 2^21 incoherent rays scaled by 8 to the 2^24 rays of a bench launch
TRAFFIC = {"raycast_incoherent": 27.79e9, "render": 47.01e9}
COHERENT_SIDE = 4096


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


def dist_env():
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0"))


# ----------------------------------------------------------------------------- workloads

def render_scene():
    from filianore_b200 import scenes
    return scenes.procedural_spheres(64, 128, 65, RENDER["width"], RENDER["height"])  # 1,048,578 triangles


def raycast_inputs(rank):
    from filianore_b200 import scenes
    tris = scenes.triangle_soup(N_TRI, seed=1)
    org, dirs = scenes.incoherent_rays(N_RAYS, seed=2 + rank)
    return tris, org, dirs


def cpu_render(steps, warmup, stride=64):
    """The oracle's integrator (hero wavelengths, all host threads) on every `stride`-th pixel."""
    import oracle
    import filianore_b200 as fb
    from filianore_b200 import scenes
    sc = render_scene()
    tab = oracle.Tables(fb.reference_tables())
    n_pix = RENDER["width"] * RENDER["height"]
    cores = os.cpu_count() or 1
    rates, mrays = [], []
    for i in range(warmup + steps):
        pixels = np.arange(i % stride, n_pix, stride, dtype=np.uint32)
        p = scenes.render_params(RENDER["spp"], RENDER["depth"], fb.FL_SPECTRAL_HERO4)
        t0 = time.perf_counter()
        _, cnt = oracle.render(sc, tab, p, nthreads=cores, pixels=pixels)
        dt = time.perf_counter() - t0
        if i >= warmup:
            rates.append(cnt["paths"] / dt)
            mrays.append(cnt["rays"] / dt / 1e6)
    return {"value": round(statistics.mean(mrays), 3), "unit": "Mrays/s", "cores": cores, "kind": "port",
            "samples_per_s": round(statistics.mean(rates), 1),
            "sample": f"every {stride}th pixel of the {RENDER['width']}x{RENDER['height']} frame "
                      f"({n_pix // stride} pixels x {RENDER['spp']} spp per step), "
                      f"CPU oracle integrator (bit-exact restatement of the reference integrator; the scene's "
                      f"environment and sphere lights have no reference class)"}


def cpu_raycast(steps, warmup):
    import oracle
    tris, org, dirs = raycast_inputs(0)
    t0 = time.perf_counter()
    bvh = oracle.CpuBVH(tris)
    build_s = time.perf_counter() - t0
    cores = os.cpu_count() or 1
    sample = min(1 << 20, N_RAYS)
    times = []
    for i in range(warmup + steps):
        sl = slice((i * sample) % N_RAYS, (i * sample) % N_RAYS + sample)
        t0 = time.perf_counter()
        bvh.trace(org[sl], dirs[sl], nthreads=cores)
        if i >= warmup:
            times.append(time.perf_counter() - t0)
    return {"value": round(sample / statistics.mean(times) / 1e6, 3), "unit": "Mrays/s", "cores": cores,
            "kind": "port",
            "sample": f"{sample} of the {N_RAYS} incoherent rays per step against the full {N_TRI}-triangle soup "
                      f"(oracle binned-SAH BVH, build {build_s:.1f} s not timed)"}


def serve_requests(n_req=200, seed=5):
    """Config-4 requests: each draws its own procedural scene (triangle count log-uniform in
    [10k, 4M]), a resolution in {128^2, 256^2, 512^2, 1024^2} and spp log-uniform in [1, 256]."""
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n_req):
        target = float(np.exp(rng.uniform(np.log(1e4), np.log(4e6))))
        res = int(rng.choice([128, 256, 512, 1024]))
        spp = max(1, int(round(float(np.exp(rng.uniform(0.0, np.log(256.0)))))))
        reqs.append((target, res, spp, 1000 + i))
    return reqs


def gpu_serve(args, world, rank, local, barrier, reduce_max):
    """200 requests at 80% of the measured one-job-at-a-time capacity (Poisson arrivals), each
    with its own scene: the continuous-batching server against the plain GPU path serving one
    job at a time (scene upload + BVH build + render per request, as the server must). The
    requests' scenes are made on the host before the clock starts (a client brings its scene
    with its request); the server's own work from fl_server_add_scene on is timed."""
    import threading
    import filianore_b200 as fb
    from filianore_b200 import scenes
    rng = np.random.default_rng(7)
    reqs = serve_requests()
    n_req = len(reqs)
    libs = {(128, 65): scenes.sphere_library(128, 65), (32, 17): scenes.sphere_library(32, 17)}
    made = [scenes.request_scene(target, sd, res, res, libs) for (target, res, _, sd) in reqs]
    ctx = fb.Context(local)
    # plain GPU path, one job at a time: service time of every request (upload, build, render)
    warm = ctx.scene(made[0])
    warm.render(scenes.render_params(1, 16), camera=warm.src.camera_struct(64, 64))
    warm.close()
    # each request's service time is the shorter of two measurements (a one-off stall, such
    # as the first use of a pool block, does not count against the serial path)
    service = [float("inf")] * n_req
    tris = [sc.n_tri for sc in made]
    samples = sum(res * res * spp for (_, res, spp, _) in reqs)
    for _ in range(2):
        for i, (target, res, spp, _) in enumerate(reqs):
            t0 = time.perf_counter()
            h = ctx.scene(made[i])
            h.render(scenes.render_params(spp, 16, fb.FL_SPECTRAL_HERO4))
            h.close()
            service[i] = min(service[i], time.perf_counter() - t0)
    mean_s = float(np.mean(service))
    lam = 0.8 / mean_s
    arrivals = np.cumsum(rng.exponential(1.0 / lam, n_req))
    arrivals -= arrivals[0]
    # serial FIFO with the measured service times
    t, serial_tti = 0.0, []
    for a, s_ in zip(arrivals, service):
        start = max(a, t)
        t = start + s_
        serial_tti.append(t - a)
    serial_makespan = t
    budget = 12 << 30
    p = lambda v, q: float(np.percentile(np.asarray(v) * 1e3, q))  # noqa: E731
    detail = {"arrival_ms": [round(a * 1e3, 2) for a in arrivals], "service_ms": [round(x * 1e3, 2) for x in service],
              "serial_tti_ms": [round(x * 1e3, 2) for x in serial_tti], "samples": [r * r * k for (_, r, k, _) in reqs],
              "tris": tris, "policies": {}}

    def mem_available_kb():
        try:
            with open("/proc/meminfo") as f:
                return int(next(l for l in f if l.startswith("MemAvailable")).split()[1])
        except (OSError, StopIteration, ValueError):
            return None

    if args.serve_detail:
        os.environ["FL_SERVE_TRACE"] = args.serve_detail + ".trace.csv"

    def run_server(name, policy):
        mem0 = mem_available_kb()
        srv = fb.Server(ctx, budget_bytes=budget, max_depth=16, max_jobs=64, max_lights=4, policy=policy,
                        wave_paths=args.serve_wave_paths)
        job_ids = [None] * n_req
        submitted = [threading.Event() for _ in range(n_req)]
        late = [0.0] * n_req
        t_start = time.perf_counter()

        def submitter():
            for i, (_, res, spp, _) in enumerate(reqs):
                sc = made[i]
                delay = arrivals[i] - (time.perf_counter() - t_start)
                if delay > 0:
                    time.sleep(delay)
                late[i] = max(0.0, time.perf_counter() - t_start - arrivals[i])
                sid = srv.add_scene(sc)
                job_ids[i] = srv.submit(sid, sc.camera_struct(res, res), scenes.render_params(spp, 16, fb.FL_SPECTRAL_HERO4))
                srv.remove_scene(sid)  # released once its job is done
                submitted[i].set()
        th = threading.Thread(target=submitter)
        th.start()
        tti, rows = [], []
        last_done, first_submit = 0.0, None
        for i in range(n_req):
            submitted[i].wait()
            _, _, st = srv.wait(job_ids[i], timeout_ms=120000)
            tti.append((st["done_ms"] - st["submit_ms"]) / 1e3 + late[i])  # from the scheduled arrival
            rows.append((tti[-1], i, st))
            last_done = max(last_done, st["done_ms"])
            first_submit = st["submit_ms"] if first_submit is None else min(first_submit, st["submit_ms"])
        th.join()
        sstats = srv.stats()
        srv.close()
        detail["policies"][name] = {"tti_ms": [round(x * 1e3, 2) for x in tti], "late_ms": [round(x * 1e3, 2) for x in late],
                                    "queued_ms": [round(st["start_ms"] - st["submit_ms"], 2) for _, _, st in rows],
                                    "mem_available_kb": [mem0, mem_available_kb()]}
        rows.sort(key=lambda r: -r[0])
        slowest = [{"req": i, "samples": st["samples"], "tris": tris[i], "res": reqs[i][1], "spp": reqs[i][2],
                    "queued_ms": round(st["start_ms"] - st["submit_ms"], 1), "tti_ms": round(t_ * 1e3, 1),
                    "alone_ms": round(service[i] * 1e3, 1)} for t_, i, st in rows[:4]]
        makespan = (last_done - first_submit) / 1e3
        return {"p50_ms": round(p(tti, 50), 2), "p99_ms": round(p(tti, 99), 2),
                "samples_per_s": round(samples / makespan, 1), "max_submit_lateness_ms": round(max(late) * 1e3, 2),
                "server": sstats, "slowest": slowest}

    policies = (("response_ratio", fb.FL_SERVE_RESPONSE_RATIO), ("first_come_lane", fb.FL_SERVE_FIRST_COME_LANE),
                ("deadline", fb.FL_SERVE_DEADLINE), ("shortest_first", fb.FL_SERVE_SHORTEST_FIRST),
                ("first_come", fb.FL_SERVE_FIRST_COME))
    if args.serve_policies:
        policies = tuple(x for x in policies if x[0] in args.serve_policies.split(","))
    results = {name: run_server(name, pol) for name, pol in policies}
    ctx.close()
    if args.serve_detail:
        with open(args.serve_detail, "w") as f:
            json.dump(detail, f)
    best = results.get("response_ratio", next(iter(results.values())))
    return {"metric": "p99 time-to-image", "value": best["p99_ms"], "unit": "ms", "n_gpus": world,
            "steps": n_req, "warmup": 1, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": "serve: 200 Poisson requests at 80% of the measured one-job-at-a-time capacity; "
                                   "each request brings its own procedural sphere scene with a triangle count "
                                   "log-uniform in [10k, 4M] (uploaded, built and released per request); "
                                   "resolution in {128^2..1024^2}; spp log-uniform in [1, 256]; depth 16; "
                                   "hero wavelengths; policy highest response ratio next; scenes built on a "
                                   "builder thread while the waves of other jobs run",
                       "scene_tris_min_median_max": [int(min(tris)), int(np.median(tris)), int(max(tris))],
                       "memory_budget_bytes": budget, "arrival_rate_per_s": round(lam, 3), "parallelism": "1 GPU"},
            "p50_ms": best["p50_ms"], "p99_ms": best["p99_ms"], "samples_per_s": best["samples_per_s"],
            "serial": {"p50_ms": round(p(serial_tti, 50), 2), "p99_ms": round(p(serial_tti, 99), 2),
                       "samples_per_s": round(samples / serial_makespan, 1),
                       "mean_service_ms": round(mean_s * 1e3, 3)},
            "policies": results}


def gpu_guide(args, world, rank, local, barrier, reduce_max):
    """Learned path guiding on the caustic scene (1024 x 1024; glass sphere of 65,536
    triangles under a sphere light of radius 0.02 and radiance 5e3; Lambert room of 12
    triangles, albedo 0.7; max depth 8, hero wavelengths): the plain GPU path at 256 spp
    (--spp) against guided renders given a fraction of its wall time (training online during
    the first 25% of each budget, passes of 4 spp), errors against a 4096-spp FP64 plain
    render. The error is also split into the caustic region (the brightest 3% of the
    reference) and the rest, with the mean radiance of the rest."""
    import filianore_b200 as fb
    from filianore_b200 import scenes
    R = RENDER["width"] if args.size else 1024
    depth = 8
    sc = scenes.caustic(R, R)
    ctx = fb.Context(local)
    s = ctx.scene(sc)
    n_ref = 4096
    n_plain = args.spp if args.spp else 256
    ref = np.zeros((R, R, 3), np.float64)
    _, rst = s.render(scenes.render_params(n_ref, depth, fb.FL_SPECTRAL_HERO4, sample_offset=1 << 24), film_xyz64=ref)
    ref /= n_ref
    lum = ref[..., 1]
    region = lum >= np.quantile(lum, 0.97)

    def errors(img, spp):
        e = np.mean((img / spp - ref) ** 2, axis=2)
        return {"mse": float(e.mean()), "mse_caustic_region": float(e[region].mean()),
                "mse_rest": float(e[~region].mean()), "mean_rest": float((img[~region] / spp).mean())}
    plain = np.zeros((R, R, 3), np.float64)
    s.render(scenes.render_params(4, depth, fb.FL_SPECTRAL_HERO4, sample_offset=1 << 22))  # warm-up
    t0 = time.perf_counter()
    _, pst = s.render(scenes.render_params(n_plain, depth, fb.FL_SPECTRAL_HERO4), film_xyz64=plain)
    t_plain = (time.perf_counter() - t0) * 1e3
    e_plain = errors(plain, n_plain)
    runs = []
    for frac in (1 / 3, 1 / 2, 1.0):
        g = fb.Guide(ctx, seed=5, learning_rate=1e-3, select_prob=0.5, batch=32768, max_records=1 << 21,
                     steps_per_wave=64, weight_average=0.99, learn_select=not args.fixed_select,
                     train_kernel=fb.FL_GUIDE_TRAIN_TCGEN05 if args.guide_tcgen05 else fb.FL_GUIDE_TRAIN_MMA_SYNC)
        img = np.zeros((R, R, 3), np.float64)
        t0 = time.perf_counter()
        _, gst = g.render_timed(s, scenes.render_params(4, depth, fb.FL_SPECTRAL_HERO4, sample_offset=1 << 20),
                                budget_ms=frac * t_plain, train_fraction=0.25, film_xyz64=img)
        wall = (time.perf_counter() - t0) * 1e3
        spp = gst["paths"] // (R * R)
        run = {"budget_frac": round(frac, 4), "wall_ms": round(wall, 1), "spp": int(spp),
               "adam_steps": g.info()["adam_steps"]}
        run.update(errors(img, spp))
        if frac == 1.0:
            # the trained guide at the plain render's sample count (sampling only)
            import torch
            img2 = np.zeros((R, R, 3), np.float64)
            torch.cuda.nvtx.range_push("timed")
            t0 = time.perf_counter()
            g.render(s, scenes.render_params(n_plain, depth, fb.FL_SPECTRAL_HERO4, sample_offset=1 << 21),
                     fb.FL_GUIDE_SAMPLE, film_xyz64=img2)
            eq = {"wall_ms": round((time.perf_counter() - t0) * 1e3, 1)}
            torch.cuda.nvtx.range_pop()
            eq.update(errors(img2, n_plain))
            run["trained_equal_spp"] = eq
        runs.append(run)
        g.close()
    ok = [r for r in runs if r["mse"] <= e_plain["mse"]]
    t_match = min(r["wall_ms"] for r in ok) if ok else None
    s.close()
    ctx.close()
    equal_time = runs[-1]
    return {"metric": f"guided wall time to the plain {n_plain}-spp MSE / plain wall time",
            "value": round(t_match / t_plain, 4) if t_match else None, "unit": "ratio", "n_gpus": world,
            "steps": len(runs), "warmup": 1, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 render, f16 weights / f32 accumulate", "data": "synthetic",
            "config": {"workload": f"guide: caustic scene {R}x{R}, glass sphere 65,536 tris, sphere light r 0.02 "
                                   f"L 5e3, depth {depth}; MLP 80-64x4-41 (8 vMF lobes + selection logit), Adam lr "
                                   "1e-3 on batches of 32 K records, weight average 0.99, one-sample MIS with "
                                   + ("c 0.5" if args.fixed_select else "c learned per point in [0.2, 0.7]")
                                   + ", training in the first "
                                   "25% of each budget",
                       "reference_spp": n_ref, "parallelism": "1 GPU"},
            "plain": dict(spp=n_plain, wall_ms=round(t_plain, 1), device_ms=round(pst["ms"], 1), **e_plain),
            "guided": runs, "equal_time_mse_ratio": round(e_plain["mse"] / equal_time["mse"], 3),
            "reference": {"spp": n_ref, "device_ms": round(rst["ms"], 1), "mean_rest": float(ref[~region].mean())}}


def config_of(workload, world):
    if workload == "render":
        W, H, spp = RENDER["width"], RENDER["height"], RENDER["spp"]
        return {"workload": "render: procedural 1,048,578-triangle scene (64 displaced spheres, Lambert / GGX "
                            f"conductor / rough dielectric, environment + sphere light), {W}x{H}, {spp} spp, "
                            "max depth 16, 4 hero wavelengths",
                "n_tri": 1048578, "width": W, "height": H, "spp": spp, "max_depth": 16,
                "l2": "working set larger than L2 (no flush)", "parallelism": f"sample split x{world}"}
    return {"workload": f"raycast: 8,388,608-triangle soup, {N_RAYS:,} incoherent rays (value) and "
                        f"{COHERENT_SIDE}x{COHERENT_SIDE} coherent primary rays, closest hit",
            "n_tri": N_TRI, "rays_per_gpu": N_RAYS, "l2": "inputs larger than L2 (no flush)",
            "parallelism": f"replicas x{world}"}


# ----------------------------------------------------------------------------- GPU arms

def gpu_render(args, world, rank, local, barrier, reduce_max):
    import torch
    import filianore_b200 as fb
    from filianore_b200 import dist as fdist, scenes
    sc = render_scene()
    ctx = fb.Context(local)
    scene = ctx.scene(sc)
    info = scene.info()
    W, H = RENDER["width"], RENDER["height"]
    film = torch.zeros((H, W, 3), dtype=torch.float32, device="cuda")
    xyz = torch.zeros((H, W, 3), dtype=torch.float64, device="cuda")

    def params(flags=0, offset=0):
        return scenes.render_params(RENDER["spp"], RENDER["depth"], fb.FL_SPECTRAL_HERO4, sample_offset=offset,
                                    flags=flags)

    def frame(p):
        _, st = scene.render(p, film_rgb=film, film_xyz64=xyz, memory=fb.FL_MEM_DEVICE)
        if world > 1:
            fdist.reduce_film(xyz, dst=0)
        return st

    for _ in range(args.warmup):
        frame(params(offset=fdist.rank_sample_offset(rank, RENDER["spp"])))
    # traversal work of one frame (instrumented, untimed)
    cstats = frame(params(fb.FL_RENDER_COUNT, fdist.rank_sample_offset(rank, RENDER["spp"])))
    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("timed")
    t_start.record()
    stats = []
    # the last timed frame also times every kernel launch with CUDA events (roofline); the
    # others replay the per-wave CUDA graph
    for k in range(args.steps):
        flags = fb.FL_RENDER_PROFILE if k == args.steps - 1 else 0
        stats.append(frame(params(flags, fdist.rank_sample_offset(rank, RENDER["spp"]))))
    t_end.record()
    torch.cuda.nvtx.range_pop()
    barrier()
    clk = clocks.stop()
    dev_ms = sum(s["ms"] for s in stats)               # device time of the renders (library events)
    wall_ms = t_start.elapsed_time(t_end)              # includes the film reduce for N > 1
    total_ms = reduce_max(max(dev_ms, wall_ms))
    rays = sum(s["rays"] for s in stats)
    paths = sum(s["paths"] for s in stats)
    value = world * rays / (total_ms / 1e3) / 1e6
    samples_per_s = world * paths / (total_ms / 1e3)

    # end to end through the C ABI, every step: the scene's triangles and material ids are
    # uploaded from pinned host memory and its BVH is built (fl_scene_create), the frame is
    # rendered, and the linear RGB film is read back into pinned host memory
    pinned = scenes.Scene(torch.from_numpy(sc.verts).pin_memory().numpy(),
                          torch.from_numpy(sc.tri_material).pin_memory().numpy(), sc.materials, sc.lights, sc.camera)
    host_film = torch.zeros((H, W, 3), dtype=torch.float32).pin_memory()
    e2e_steps = max(2, args.steps // 2)

    parts = {"scene_create_ms": 0.0, "render_call_ms": 0.0, "render_device_ms": 0.0, "scene_destroy_ms": 0.0}

    def e2e_step():
        t0 = time.perf_counter()
        h = ctx.scene(pinned)
        t1 = time.perf_counter()
        _, st = h.render(params(offset=fdist.rank_sample_offset(rank, RENDER["spp"])), film_rgb=host_film.numpy(), memory=fb.FL_MEM_HOST)
        t2 = time.perf_counter()
        h.close()
        t3 = time.perf_counter()
        parts["scene_create_ms"] += (t1 - t0) * 1e3
        parts["render_call_ms"] += (t2 - t1) * 1e3
        parts["render_device_ms"] += st["ms"]
        parts["scene_destroy_ms"] += (t3 - t2) * 1e3
        return st
    e2e_step()
    for k in parts:
        parts[k] = 0.0
    barrier()
    t0 = time.perf_counter()
    e_rays = 0
    for _ in range(e2e_steps):
        e_rays += e2e_step()["rays"]
    barrier()
    e2e_s = reduce_max(time.perf_counter() - t0)
    e2e = {"value": round(world * e_rays / e2e_s / 1e6, 3), "unit": "Mrays/s",
           "samples_per_s": round(world * e2e_steps * W * H * RENDER["spp"] / e2e_s, 1),
           "h2d_bytes_per_step": int(pinned.verts.nbytes + pinned.tri_material.nbytes),
           "d2h_bytes_per_step": W * H * 3 * 4,
           "note": "per step: scene upload from pinned host memory + BVH build + render + film readback",
           "breakdown_ms_per_step": {k: round(v / e2e_steps, 2) for k, v in parts.items()}}

    peaks = load_peaks()
    prof = stats[-1]
    trav_ms = prof["ms_trace"] + prof["ms_shadow"]
    alg_bytes = cstats["rays"] * (RAY_BYTES + HIT_BYTES) + NODE_BYTES * cstats["nodes_visited"] + \
        TRI_BYTES * cstats["tris_tested"]
    achieved = alg_bytes / (trav_ms / 1e3) / 1e9
    share = {k: round(prof[f"ms_{k}"] / prof["ms"], 4) for k in ("trace", "shade", "shadow", "continue")}
    full = RENDER["width"] == 1920 and RENDER["height"] == 1080 and RENDER["spp"] == 64
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": TRAFFIC["render"] if full else None,
                "traffic_unit": "bytes per frame (ncu, every traversal launch of one frame)", "peak_src": peaks["src"],
                "kernel": "BVH traversal (k_trace_paths + k_trace_rays2)",
                "alg_bytes_per_frame": int(alg_bytes), "traversal_ms_per_frame": round(trav_ms, 3),
                "profiled_frame_ms": round(prof["ms"], 3),
                "nodes_per_ray": round(cstats["nodes_visited"] / cstats["rays"], 2),
                "tris_per_ray": round(cstats["tris_tested"] / cstats["rays"], 2), "time_share": share}
    line = {"metric": "Mrays/s", "value": round(value, 3), "unit": "Mrays/s", "samples_per_s": round(samples_per_s, 1),
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(total_ms / args.steps, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config_of("render", world),
            "roofline": roofline, "e2e": e2e, "gpu_launches": sum(s["launches"] for s in stats), "clocks": clk,
            "rays_per_frame": stats[0]["rays"], "paths_per_frame": stats[0]["paths"],
            "bvh": {"nodes": info["n_nodes"], "depth": info["max_depth"], "build_ms": round(info["build_ms"], 2),
                    "bytes": info["bvh_bytes"]}}
    scene.close()
    ctx.close()
    if not args.no_raycast:
        # the 8,388,608-triangle ray-cast workload (both ray sets), measured in the same run
        line["raycast"] = measure_raycast(args, world, rank, local, barrier, reduce_max, max(3, args.steps))
    return line


def measure_raycast(args, world, rank, local, barrier, reduce_max, steps):
    """The ray-cast workload on one GPU: the 8,388,608-triangle soup, its BVH built on the
    device, and both ray sets (16,777,216 incoherent rays; 4096 x 4096 pinhole primary rays),
    each timed per launch with CUDA events on the launching stream. Returns per-set throughput,
    the traversal roofline (algorithmic bytes from the device visit counters of the same rays),
    and the end-to-end rate through the C ABI with host buffers."""
    import torch
    import filianore_b200 as fb
    from filianore_b200 import scenes
    tris, org, dirs = raycast_inputs(rank)
    sc = scenes.Scene(tris, np.zeros(N_TRI, np.uint32), [{"type": 0, "rgb": (0.5, 0.5, 0.5)}], [], None)
    side = COHERENT_SIDE if N_RAYS == 1 << 24 else max(64, int(N_RAYS ** 0.5))
    sets = {"incoherent": (org, dirs), "coherent": scenes.coherent_rays(side, side)}
    ctx = fb.Context(local)
    scene = ctx.scene(sc)
    info = scene.info()
    peaks = load_peaks()
    stream = torch.cuda.current_stream().cuda_stream
    L = fb.lib()
    out = {"n_tri": N_TRI, "bvh": {"nodes": info["n_nodes"], "depth": info["max_depth"],
                                   "build_ms": round(info["build_ms"], 2), "bytes": info["bvh_bytes"]}}
    e2e_rays, e2e_s = 0, 0.0
    clocks = ClockSampler(local)
    clocks.start()
    for name, (o, d) in sets.items():
        n = o.shape[0]
        d_org = torch.from_numpy(o).cuda()
        d_dir = torch.from_numpy(d).cuda()
        d_hits = torch.empty((n, 4), dtype=torch.int32, device="cuda")
        nodes, trisv = scene.trace_count(d_org, d_dir)
        alg_bytes = n * (RAY_BYTES + HIT_BYTES) + NODE_BYTES * nodes + TRI_BYTES * trisv
        for _ in range(args.warmup):
            scene.trace_closest(d_org, d_dir, out=d_hits, stream=stream)
        barrier()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        torch.cuda.nvtx.range_push(f"timed_{name}")
        for k in range(steps):
            ev[k][0].record()
            scene.trace_closest(d_org, d_dir, out=d_hits, stream=stream)
            ev[k][1].record()
        torch.cuda.nvtx.range_pop()
        barrier()
        launch_ms = reduce_max(statistics.mean(a.elapsed_time(b) for a, b in ev))
        achieved = alg_bytes / (launch_ms / 1e3) / 1e9
        mrays = n / (launch_ms / 1e3) / 1e6
        out[name] = {
            "rays": n, "mrays_s": round(world * mrays, 3), "ms_per_launch": round(launch_ms, 4),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": round(achieved / peaks["hbm_gbs"], 4), "peak_src": peaks["src"],
                         "kernel": "k_trace<closest>", "alg_bytes_per_launch": int(alg_bytes),
                         "traffic": TRAFFIC.get(f"raycast_{name}") if N_RAYS == 1 << 24 else None,
                         "traffic_unit": "bytes per launch (ncu: 2^21 rays, x 8)",
                         # layout-independent floor: only the ray read and the hit write
                         "floor_bytes_per_ray": RAY_BYTES + HIT_BYTES,
                         "floor_frac": round(n * (RAY_BYTES + HIT_BYTES) / (launch_ms / 1e3) / 1e9 / peaks["hbm_gbs"], 4)},
            "nodes_per_ray": round(nodes / n, 2), "tris_per_ray": round(trisv / n, 2)}
        # end to end through the C ABI with pinned host buffers: H2D of the rays, the trace,
        # D2H of the hits, every call
        h_org = torch.from_numpy(o).pin_memory()
        h_dir = torch.from_numpy(d).pin_memory()
        h_hits = torch.empty((n, 4), dtype=torch.int32).pin_memory()

        def host_call():
            fb.check(L.fl_trace_closest(scene.h, C.c_void_p(h_org.data_ptr()), C.c_void_p(h_dir.data_ptr()), n,
                                        C.c_void_p(h_hits.data_ptr()), fb.FL_MEM_HOST, None), ctx.h)
        host_call()
        e_steps = max(2, steps // 2)
        barrier()
        t0 = time.perf_counter()
        for _ in range(e_steps):
            host_call()
        barrier()
        dt = reduce_max((time.perf_counter() - t0) / e_steps)
        out[name]["e2e_mrays_s"] = round(world * n / dt / 1e6, 3)
        e2e_rays += n
        e2e_s += dt
        del d_org, d_dir, d_hits, h_org, h_dir, h_hits
    out["clocks"] = clocks.stop()
    out["e2e"] = {"value": round(world * e2e_rays / e2e_s / 1e6, 3), "unit": "Mrays/s",
                  "h2d_bytes_per_step": e2e_rays * RAY_BYTES, "d2h_bytes_per_step": e2e_rays * HIT_BYTES,
                  "note": "one step = both ray sets through fl_trace_closest with pinned host buffers"}
    scene.close()
    ctx.close()
    return out


def gpu_raycast(args, world, rank, local, barrier, reduce_max):
    rc = measure_raycast(args, world, rank, local, barrier, reduce_max, args.steps)
    inc = rc["incoherent"]
    line = {"metric": "Mrays/s", "value": inc["mrays_s"], "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": inc["ms_per_launch"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_of("raycast", world), "roofline": inc["roofline"],
            "e2e": {"value": inc["e2e_mrays_s"], "unit": "Mrays/s", "h2d_bytes_per_step": inc["rays"] * RAY_BYTES,
                    "d2h_bytes_per_step": inc["rays"] * HIT_BYTES},
            "gpu_launches": args.steps, "clocks": rc["clocks"], "coherent": rc["coherent"], "bvh": rc["bvh"],
            "nodes_per_ray": inc["nodes_per_ray"], "tris_per_ray": inc["tris_per_ray"]}
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="render", choices=["render", "raycast", "serve", "guide"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve-detail", default=None, help="serve: write per-request times to this JSON file")
    ap.add_argument("--serve-wave-paths", type=int, default=0, help="serve: the server's path slots (0: its default)")
    ap.add_argument("--serve-policies", default=None, help="serve: comma-separated subset of the policies")
    ap.add_argument("--no-raycast", action="store_true", help="render: skip the ray-cast sub-measurement")
    ap.add_argument("--guide-tcgen05", action="store_true", help="guide: train with the tcgen05 kernel")
    ap.add_argument("--fixed-select", action="store_true",
                    help="guide: a fixed selection probability c = 0.5 instead of the learned one")
    ap.add_argument("--size", default=None, help="render: WxH (smaller cases for profiling)")
    ap.add_argument("--spp", type=int, default=None, help="render: samples per pixel")
    ap.add_argument("--rays", type=int, default=None, help="raycast: rays per batch")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    global N_RAYS
    if args.size:
        RENDER["width"], RENDER["height"] = (int(v) for v in args.size.lower().split("x"))
    if args.spp:
        RENDER["spp"] = args.spp
    if args.rays:
        N_RAYS = args.rays
    world, rank, local = dist_env()

    if args.impl == "reference":
        if rank == 0:
            cb = cpu_render(args.steps, args.warmup) if args.workload == "render" else cpu_raycast(args.steps, args.warmup)
            line = {"metric": "Mrays/s", "value": cb["value"], "unit": "Mrays/s", "n_gpus": world,
                    "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                    "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                    "config": config_of(args.workload, world), "impl": "reference", "cpu_baseline": cb,
                    "e2e": {"value": cb["value"], "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                            "d2h_bytes_per_step": 0}}
            if "samples_per_s" in cb:
                line["samples_per_s"] = cb["samples_per_s"]
            print(json.dumps(line), flush=True)
        return

    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    def reduce_max(x):
        if world == 1:
            return x
        import torch.distributed as dist
        t = torch.tensor([float(x)], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    run = {"render": gpu_render, "raycast": gpu_raycast, "serve": gpu_serve, "guide": gpu_guide}[args.workload]
    line = run(args, world, rank, local, barrier, reduce_max)
    if rank == 0:
        if not args.no_cpu_baseline and args.workload in ("render", "raycast"):
            line["cpu_baseline"] = (cpu_render(2, 0) if args.workload == "render" else cpu_raycast(3, 1))
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
