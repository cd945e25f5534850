"""Full-size workloads of configs 1-3 and 5, used by bench.py.

Each function builds its seeded synthetic scene (renderbox2_b200.configs),
runs on the current CUDA device and returns a dict of measurements.  Times
are CUDA-event times on the launching stream unless marked wall-clock.
"""
from __future__ import annotations

import time

import numpy as np


def _event_ms(fn, stream, reps=1):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def integrator(kind: str, warmup: int = 1, keep: dict | None = None, node_order: int | None = None,
               tri_cost: float | None = None, node_threshold: int = 0):
    """Config 1 (AO), 2 (PT) or 3 (BDPT) at full size: samples/s and Mrays/s.
    "raycast": the config-2 scene, camera and spp through the ray-cast
    integrator (primary rays only, primitive-id shading).
    `keep` (optional dict) receives the scene, BVH and config used.  The
    traversal layout is `node_order`, or (None) the faster of the binary BFS
    and the compressed 8-wide layout on one timed frame each.  The BVH is
    built with the benchmark SAH costs (configs.BUILD; `tri_cost` overrides
    the triangle cost).  `node_threshold` sets the traversal's node-phase
    threshold (rb2_launch_config.node_threshold; 0: the layout's default)."""
    import torch

    import renderbox2_b200 as rb
    from renderbox2_b200 import configs
    from renderbox2_b200.render import (AmbientOcclusionIntegratorParams, BidirectionalPathIntegratorLvcParams,
                                        DeviceScene, Integrator, PathIntegratorParams, RayCastIntegratorParams)
    t0 = time.time()
    if kind == "ao":
        c = configs.CONFIG1
        scene = rb.heightfield_scene(seed=c["seed"], grid_n=c["grid_n"], amplitude=c["amplitude"],
                                     n_boxes=c["n_boxes"], box_min=c["box_min"], box_max=c["box_max"])
    else:
        c = configs.CONFIG2 if kind in ("pt", "raycast") else configs.CONFIG3
        scene = rb.RoomScene(seed=c["seed"], n_boxes=c["n_boxes"], n_spheres=c["n_spheres"],
                             sphere_subdiv=c["sphere_subdiv"], rmin=c["rmin"], rmax=c["rmax"],
                             n_lights=c["n_lights"], emission=c["emission"], room_size=c["room_size"])
    from renderbox2_b200.accel import Platform
    tri_cost = configs.BUILD["sah_triangle_cost"] if tri_cost is None else tri_cost
    bvh = rb.BVH(scene, platform=Platform(sah_node_cost=configs.BUILD["sah_node_cost"], sah_triangle_cost=tri_cost))
    build_s = time.time() - t0
    tracer = rb.CudaTracer(bvh)
    it = Integrator(tracer, DeviceScene(scene))
    it.set_timing(True)  # traversal launches bracketed by CUDA events (stats "trace_ms")
    if node_threshold:
        it.set_launch(node_threshold=node_threshold)
    scale = c.get("room_size", 1.0)
    eye = [x * scale for x in c["eye"]]
    look = [x * scale for x in c["lookat"]]
    cam = rb.PerspectiveCamera(eye, look, c["up"], (c["width"], c["height"]), c["fov"])
    stream = torch.cuda.Stream()
    npix = c["width"] * c["height"]
    with torch.cuda.stream(stream):
        if kind == "ao":
            p = AmbientOcclusionIntegratorParams(samples=c["ao_samples"], radius=c["ao_radius"], seed=c["ao_seed"])
            out = torch.empty((npix,), dtype=torch.float32, device="cuda")
            run = lambda: it.render_ao(cam, p, out=out, stream=stream)  # noqa: E731
            samples = npix * c["ao_samples"]
        elif kind == "pt":
            p = PathIntegratorParams(spp=c["spp"], max_depth=c["max_depth"], rr_start=c["rr_start"],
                                     rr_prob=c["rr_prob"], seed=1)
            out = torch.empty((npix, 3), dtype=torch.float32, device="cuda")
            run = lambda: it.render_pt(cam, p, out=out, stream=stream)  # noqa: E731
            samples = npix * c["spp"]
        elif kind == "raycast":
            p = RayCastIntegratorParams("primitive_id", spp=c["spp"], seed=1)
            out = torch.empty((npix, 3), dtype=torch.float32, device="cuda")
            run = lambda: it.render_raycast(cam, p, out=out, stream=stream)  # noqa: E731
            samples = npix * c["spp"]
        else:
            p = BidirectionalPathIntegratorLvcParams(spp=c["spp"], max_path_length=c["max_path_length"],
                                                     connections=c["lvc_connections"], seed=1)
            out = torch.empty((npix, 3), dtype=torch.float32, device="cuda")
            run = lambda: it.render_bdpt(cam, p, out=out, stream=stream)  # noqa: E731
            samples = npix * c["spp"]
        orders = [node_order] if node_order is not None else [rb.NODE_ORDER_BFS, rb.NODE_ORDER_CW8]
        probe = {}
        for o in orders:
            tracer.set_node_order(o)
            run()
            torch.cuda.synchronize()
            if len(orders) > 1:
                probe[o] = _event_ms(run, stream)
        if probe:
            tracer.set_node_order(min(probe, key=probe.get))
        for _ in range(warmup):
            run()
        torch.cuda.synchronize()
        ms = _event_ms(run, stream)
    st = it.stats(stream)
    if keep is not None:
        keep.update(scene=scene, bvh=bvh, config=c, eye=eye, lookat=look)
    rays = (npix if kind == "ao" else 0) + sum(st[k] for k in ("primary_rays", "extension_rays", "shadow_rays",
                                                              "connection_rays", "light_rays"))
    if kind == "ao":
        rays = npix + npix * c["ao_samples"]
    return {"workload": kind, "triangles": scene.num_triangles, "width": c["width"], "height": c["height"],
            "samples": int(samples), "ms": round(ms, 3), "samples_per_s": round(samples / (ms / 1e3), 1),
            "mrays_per_s": round(rays / (ms / 1e3) / 1e6, 2), "rays": int(rays), "build_s": round(build_s, 2),
            "sah_triangle_cost": tri_cost,
            "stats": st, "image_mean": float(out.float().mean().item()),
            "node_order": {0: "dfs", 1: "bfs", 2: "wide4", 3: "cw8"}[tracer.node_order()],
            "layout_probe_ms": {str(k): round(v, 3) for k, v in probe.items()}}


def serving(n_jobs: int = 10000, n_bvh: int = 32, seed: int = 5, slots: int = 32, burst_jobs: int = 2000,
            shared: bool | None = None, hbm_budget: int = 48 << 30):
    """Config 5: pool of n_bvh lit heightfields (1k..4M triangles,
    log-uniform), n_jobs jobs, 70 % tile renders / 30 % ray batches.  The
    arrival rate is the throughput of the plain path (one job at a time) on a
    burst of the first `burst_jobs` jobs, i.e. the rate that saturates it;
    both paths then serve the same Poisson arrival sequence of all n_jobs.
    `capacity` compares both paths on that burst (every job queued at t = 0).
    The continuous server runs `slots` concurrent jobs whose admitted
    working sets stay within `hbm_budget` bytes.
    `shared` (default: more than 1000 jobs) takes ray-job inputs from one
    pinned ray set per BVH and outputs from a circular pinned arena
    (serve.SharedBuffers) instead of per-job host buffers."""
    from renderbox2_b200 import configs
    from renderbox2_b200.serve import (Server, SharedBuffers, build_pool, config5_jobs, pool_triangle_counts,
                                       poisson_arrivals)
    c = configs.CONFIG5
    t0 = time.time()
    counts = pool_triangle_counts(n_bvh, c["tri_min"], c["tri_max"], seed)
    pool = build_pool(counts, seed=seed)
    use_shared = n_jobs > 1000 if shared is None else shared
    sh = SharedBuffers(pool, rays_per_bvh=c["rays_max"]) if use_shared else None
    jobs = config5_jobs(pool, n_jobs, seed=seed, shared=sh)
    setup_s = time.time() - t0
    cont = Server(pool, slots=slots, fifo=False, hbm_budget=hbm_budget)
    plain = Server(pool, fifo=True)
    # warm-up: a few jobs through both
    cont.run(jobs.subset(range(min(8, n_jobs))))
    plain.run(jobs.subset(range(min(8, n_jobs))))
    nb = min(burst_jobs, n_jobs)
    _, burst = plain.run(jobs.subset(range(nb)))
    _, cburst = cont.run(jobs.subset(range(nb)))
    rate = nb / burst["wall_s"]
    arr = poisson_arrivals(n_jobs, rate, seed=seed + 1)
    _, s_plain = plain.run(jobs.with_arrivals(arr))
    _, s_cont = cont.run(jobs.with_arrivals(arr))
    keep = ("p50_s", "p99_s", "mean_s", "mrays_per_s", "wall_s", "max_concurrent")
    return {"jobs": n_jobs, "burst_jobs": nb, "slots": slots, "hbm_budget_gb": hbm_budget >> 30,
            "host_buffers": "shared ray sets + output arena" if use_shared
            else "per job", "bvhs": n_bvh, "pool_triangles": int(sum(counts)),
            "arrival_rate_jobs_per_s": round(rate, 2), "setup_s": round(setup_s, 1),
            "resident_gb": round(s_cont["resident_bytes"] / 1e9, 2),
            "continuous": {k: round(s_cont[k], 5) for k in keep},
            "plain_fifo": {k: round(s_plain[k], 5) for k in keep},
            "p99_speedup": round(s_plain["p99_s"] / max(s_cont["p99_s"], 1e-9), 3),
            "throughput_ratio": round(s_cont["mrays_per_s"] / max(s_plain["mrays_per_s"], 1e-9), 3),
            "capacity": {"note": "all jobs queued at t = 0 (burst): rays / makespan",
                         "continuous_mrays_per_s": round(cburst["mrays_per_s"], 1),
                         "plain_fifo_mrays_per_s": round(burst["mrays_per_s"], 1),
                         "ratio": round(cburst["mrays_per_s"] / max(burst["mrays_per_s"], 1e-9), 3)}}


def serving_curve(n_jobs: int = 3000, n_bvh: int = 32, seed: int = 5, slots: int = 32,
                  loads=(0.5, 0.8, 1.0, 1.2), burst_jobs: int = 1000, hbm_budget: int = 48 << 30):
    """Latency against offered load for config 5: the continuous server's
    burst capacity (jobs per second with every job queued at t = 0) sets the
    unit of load; each point serves the same n_jobs with Poisson arrivals at
    load x that rate, through the continuous server and the one-at-a-time
    FIFO server.  Returns the capacity and one record per load."""
    from renderbox2_b200 import configs
    from renderbox2_b200.serve import (Server, SharedBuffers, build_pool, config5_jobs, pool_triangle_counts,
                                       poisson_arrivals)
    c = configs.CONFIG5
    counts = pool_triangle_counts(n_bvh, c["tri_min"], c["tri_max"], seed)
    pool = build_pool(counts, seed=seed)
    sh = SharedBuffers(pool, rays_per_bvh=c["rays_max"])
    jobs = config5_jobs(pool, n_jobs, seed=seed, shared=sh)
    cont = Server(pool, slots=slots, fifo=False, hbm_budget=hbm_budget)
    plain = Server(pool, fifo=True)
    cont.run(jobs.subset(range(min(8, n_jobs))))
    plain.run(jobs.subset(range(min(8, n_jobs))))
    nb = min(burst_jobs, n_jobs)
    _, cb = cont.run(jobs.subset(range(nb)))
    _, pb = plain.run(jobs.subset(range(nb)))
    cap = nb / cb["wall_s"]
    out = {"jobs": n_jobs, "slots": slots, "continuous_capacity_jobs_per_s": round(cap, 2),
           "plain_capacity_jobs_per_s": round(nb / pb["wall_s"], 2),
           "capacity_ratio_mrays": round(cb["mrays_per_s"] / max(pb["mrays_per_s"], 1e-9), 3), "points": []}
    for k, load in enumerate(loads):
        arr = poisson_arrivals(n_jobs, load * cap, seed=seed + 10 + k)
        _, sc = cont.run(jobs.with_arrivals(arr))
        _, sp = plain.run(jobs.with_arrivals(arr))
        out["points"].append({
            "load": load, "arrival_rate_jobs_per_s": round(load * cap, 2),
            "continuous": {"p50_s": round(sc["p50_s"], 5), "p99_s": round(sc["p99_s"], 5),
                           "mrays_per_s": round(sc["mrays_per_s"], 1)},
            "plain_fifo": {"p50_s": round(sp["p50_s"], 5), "p99_s": round(sp["p99_s"], 5),
                           "mrays_per_s": round(sp["mrays_per_s"], 1)}})
    return out
