"""Benchmark: incoherent ray-query throughput on one B200 (config 4 workload).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl rb2|reference]
                  [--rays-per-scene R] [--scenes S] [--workload trace|ao|pt|bdpt|raycast]

One step = every scene's ray batch traced once: 64 heightfield scenes with
log-uniform 1k..2M triangles, 1M incoherent diffuse-bounce rays per scene,
50 % closest-hit and 50 % any-hit (occlusion).  Inputs are resident in HBM
when the timed region starts; L2 is flushed (256 MB write) between timed
steps.  `e2e` repeats the step through the host-buffer C-ABI call
(rb2_trace_host_jobs: pinned host rays in, hits / occlusion bytes out, the
copies pipelined with traversal over several streams), copies included.  Under torchrun each rank runs the same
workload on its own GPU (replicas, no collective); `value` = all ranks' rays
/ max-over-ranks time.

--impl reference times the CPU restatement of the reference traversal (the
reference has no host traversal of its own) on all host cores over a bounded
sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mrays/s incoherent closest-hit; served-job p50/p99 vs plain launches, 1 B200"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ----------------------------------------------------------------------------- workload
def build_workload(n_scenes: int, rays_per_scene: int, seed_base: int = 4):
    import renderbox2_b200 as rb
    from renderbox2_b200.configs import CONFIG4, config4_triangle_counts
    counts = config4_triangle_counts(dict(CONFIG4, n_scenes=64))[:n_scenes]
    scenes = []
    t0 = time.time()
    build_s = 0.0
    for k, tris in enumerate(counts):
        sc = rb.heightfield_for_triangles(seed=seed_base * 1000 + k, n_tris=tris)
        tb = time.time()
        bvh = rb.BVH(sc)
        build_s += time.time() - tb
        rays, flags = rb.surface_rays(sc, seed=seed_base * 1000 + 500 + k, n=rays_per_scene,
                                      offset_scale=CONFIG4["offset_scale"],
                                      anyhit_fraction=CONFIG4["anyhit_fraction"])
        order = np.argsort(flags, kind="stable")  # closest-hit rays first, then any-hit
        rays = np.ascontiguousarray(rays[order])
        n_ch = int((flags == 0).sum())
        scenes.append(dict(scene=sc, bvh=bvh, rays=rays, n_ch=n_ch, tris=sc.num_triangles))
    log(f"workload: {n_scenes} scenes, {sum(s['tris'] for s in scenes):,} triangles, "
        f"{n_scenes * rays_per_scene:,} rays; build {build_s:.1f}s, total setup {time.time() - t0:.1f}s")
    return scenes, build_s


def oracle_bytes_sample(scenes, per_scene: int, nthreads: int = 0):
    """Canonical single-lane visit counts of the oracle on a sample of each
    scene's rays -> mean algorithmic bytes per ray, per mode and scene."""
    import oracle
    out = []
    t_cpu = 0.0
    n_cpu = 0
    for s in scenes:
        nodes, woop, tri = s["bvh"].buffers_view()
        res = {}
        for mode, sl in (("ch", slice(0, s["n_ch"])), ("ah", slice(s["n_ch"], None))):
            r = s["rays"][sl]
            idx = np.linspace(0, r.shape[0] - 1, min(per_scene, r.shape[0])).astype(np.int64)
            t0 = time.perf_counter()
            _, cnt = oracle.trace(nodes, woop, tri, r[idx], any_hit=(mode == "ah"), counts=True, nthreads=nthreads)
            t_cpu += time.perf_counter() - t0
            n_cpu += idx.size
            out_b = 16 if mode == "ch" else 1
            bpr = 32 + 64 * cnt["nodes"].astype(np.float64) + 48 * cnt["tris"] + 16 * cnt["leafterms"] + out_b
            res[mode] = dict(bytes_per_ray=float(bpr.mean()), nodes=float(cnt["nodes"].mean()),
                             tris=float(cnt["tris"].mean()))
        out.append(res)
    return out, (n_cpu / t_cpu / 1e6 if t_cpu > 0 else 0.0), n_cpu, t_cpu


# ------------------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = ROOT / "gpurun_out" / f"clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.path.parent.mkdir(exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = [r.split(",") for r in self.path.read_text().splitlines() if r.strip()]
        rows = [[c.strip() for c in r] for r in rows if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# --------------------------------------------------------------------------- GPU arm
def run_rb2(args, rank, world, local_rank):
    import torch

    import renderbox2_b200 as rb
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    scenes, build_s = build_workload(args.scenes, args.rays_per_scene)
    total_rays = sum(s["rays"].shape[0] for s in scenes)
    n_ch_total = sum(s["n_ch"] for s in scenes)
    tracers, d_rays, d_hits, d_occ = [], [], [], []
    for s in scenes:
        tracers.append(rb.CudaTracer(s["bvh"]))
        d_rays.append(torch.from_numpy(s["rays"]).to(dev))
        d_hits.append(torch.empty((s["n_ch"], 4), dtype=torch.int32, device=dev))
        d_occ.append(torch.empty((s["rays"].shape[0] - s["n_ch"],), dtype=torch.uint8, device=dev))
    bvh_bytes = sum(t.device_bytes() for t in tracers)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def ev():
        return torch.cuda.Event(enable_timing=True)

    # ---- plain path: two launches per scene (closest-hit half, any-hit half).
    pev = [[(ev(), ev()) for _ in range(2)] for _ in scenes]

    def plain_step(record: bool):
        with torch.cuda.stream(stream):
            for k, s in enumerate(scenes):
                tr, r = tracers[k], d_rays[k]
                if record:
                    pev[k][0][0].record(stream)
                tr.trace(r[: s["n_ch"]], any_hit=False, out=d_hits[k], stream=stream)
                if record:
                    pev[k][0][1].record(stream)
                    pev[k][1][0].record(stream)
                tr.trace_occlusion(r[s["n_ch"]:], out=d_occ[k], stream=stream)
                if record:
                    pev[k][1][1].record(stream)

    # ---- batched path: one persistent launch over all 2 x scenes jobs, graph-replayed.
    jobs = []
    for k, s in enumerate(scenes):
        jobs.append((tracers[k], d_rays[k][: s["n_ch"]], rb.MODE_CLOSEST, d_hits[k], None))
        jobs.append((tracers[k], d_rays[k][s["n_ch"]:], rb.MODE_OCCLUSION, d_occ[k], None))
    batch = rb.TraceBatch(jobs)

    def timed(step_fn, steps, per_step_events=None):
        """Times `steps` steps with CUDA events on the launching stream,
        flushing L2 (256 MB write) before each step outside the timed region."""
        t0, t1 = ev(), ev()
        ms = []
        for it in range(steps):
            flush.fill_(float(it))
            torch.cuda.synchronize(dev)
            t0.record(stream)
            step_fn()
            t1.record(stream)
            torch.cuda.synchronize(dev)
            ms.append(t0.elapsed_time(t1))
            if per_step_events:
                per_step_events()
        return ms

    ch_ms, ah_ms = np.zeros(len(scenes)), np.zeros(len(scenes))

    def collect_plain():
        for k in range(len(scenes)):
            ch_ms[k] += pev[k][0][0].elapsed_time(pev[k][0][1])
            ah_ms[k] += pev[k][1][0].elapsed_time(pev[k][1][1])

    # The plain path is timed first, with the tracers' defaults (the reference's
    # DFS Compact2 layout, default launch shape), before the autotuner changes
    # any tracer's layout; then the batched launch is tuned (untimed), captured
    # and timed.  Clocks are sampled across both timed regions.
    for _ in range(args.warmup):
        plain_step(False)
    torch.cuda.synchronize(dev)
    barrier(world)
    with ClockSampler(local_rank) as clk:
        plain_ms = timed(lambda: plain_step(True), args.steps, collect_plain)
        tuned, tuned_ms = batch.autotune(stream=stream, reps=5)
        batch.capture(stream)
        for _ in range(args.warmup):
            batch.launch(stream)
        torch.cuda.synchronize(dev)
        barrier(world)
        batch_ms = timed(lambda: batch.launch(stream), args.steps)
    clocks = clk.summary()
    plain_rate, plain_total = whole_job_rate(total_rays * args.steps, sum(plain_ms), world, dev)
    batch_rate, batch_total = whole_job_rate(total_rays * args.steps, sum(batch_ms), world, dev)
    for t in tracers:
        assert t.status() == 0, "device status word set"
    assert batch.status() == 0, "batch status word set"

    # ---- e2e through the host-buffer C-ABI calls (pinned host memory, copies in the timed region).
    # Headline: rb2_trace_host_jobs, chunks cycling through several streams so
    # H2D, traversal and D2H overlap.  Also reported: one blocking
    # rb2_trace_host call per job (no overlap).
    h_rays = [torch.from_numpy(s["rays"]).pin_memory() for s in scenes]
    h_hits = [torch.empty((s["n_ch"], 4), dtype=torch.int32).pin_memory() for s in scenes]
    h_occ = [torch.empty((s["rays"].shape[0] - s["n_ch"],), dtype=torch.uint8).pin_memory() for s in scenes]
    h_hits16 = [torch.empty((s["rays"].shape[0], 4), dtype=torch.int32).pin_memory() for s in scenes]
    from renderbox2_b200._native import check, lib
    L = lib()
    sh = stream.cuda_stream
    pipe = rb.HostPipeline(chunk_rays=args.e2e_chunk, depth=args.e2e_depth)
    host_jobs = []
    for k, s in enumerate(scenes):
        n_ch = s["n_ch"]
        host_jobs.append((tracers[k], h_rays[k][:n_ch], rb.MODE_CLOSEST, h_hits[k], None))
        host_jobs.append((tracers[k], h_rays[k][n_ch:], rb.MODE_OCCLUSION, h_occ[k], None))
    host_arr = pipe.job_array(host_jobs)
    h2d_bytes = int(total_rays * 32)
    d2h_bytes = int(n_ch_total * 16 + (total_rays - n_ch_total))

    def e2e_step():
        pipe.trace_jobs(host_arr, stream)

    def e2e_single_step():
        for k, s in enumerate(scenes):
            n_ch = s["n_ch"]
            hr, hh = h_rays[k], h_hits16[k]
            check(L.rb2_trace_host(tracers[k].handle, hr.data_ptr(), n_ch, 0, None, hh.data_ptr(), sh))
            check(L.rb2_trace_host(tracers[k].handle, hr.data_ptr() + 32 * n_ch, s["rays"].shape[0] - n_ch, 1, None,
                                   hh.data_ptr() + 16 * n_ch, sh))

    def device_ms(fn, steps):
        """CUDA events on `stream` around `steps` host calls (each call's
        device work, copies included, is ordered on `stream`)."""
        for _ in range(max(1, args.warmup)):
            fn()
        torch.cuda.synchronize(dev)
        barrier(world)
        t0, t1 = ev(), ev()
        t0.record(stream)
        for _ in range(steps):
            fn()
        t1.record(stream)
        torch.cuda.synchronize(dev)
        return t0.elapsed_time(t1)

    e2e_steps = max(1, min(args.steps, 5))
    e2e_single_steps = max(1, min(args.steps, 2))
    e2e_rate, _ = whole_job_rate(total_rays * e2e_steps, device_ms(e2e_step, e2e_steps), world, dev)
    e2e_single_rate, _ = whole_job_rate(total_rays * e2e_single_steps, device_ms(e2e_single_step, e2e_single_steps),
                                        world, dev)

    # ---- roofline: dominant kernel = the batched traversal launch (one per step).
    bytes_info, _, _, _ = oracle_bytes_sample(scenes, 4096)
    ch_bytes = sum(bi["ch"]["bytes_per_ray"] * s["n_ch"] for bi, s in zip(bytes_info, scenes))
    ah_bytes = sum(bi["ah"]["bytes_per_ray"] * (s["rays"].shape[0] - s["n_ch"]) for bi, s in zip(bytes_info, scenes))
    launch_s = batch_total / 1e3 / args.steps
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "MEASURED_PEAKS.json hbm_gbs (measured)" if "hbm_gbs" in peaks else "fallback 6650 GB/s"
    alg_per_launch = ch_bytes + ah_bytes
    achieved = alg_per_launch / launch_s / 1e9
    # DRAM traffic per launch: the ncu capture of the same batched kernel on
    # 8 scenes x 500k triangles with 4.19M incoherent rays, half closest hit /
    # half occlusion, measured against 7961.2 MB of algorithmic bytes: 618.5 MB
    # for the binary layout (profiles/k_trace_jobs_batched_8x500k_full.md) and
    # 445.7 MB for the compressed 8-wide layout
    # (profiles/k_trace_jobs_cw8_batched_8x500k_full.md); scaled to this launch
    # by algorithmic bytes.
    cw8 = tuned is not None and tuned.get("node_order") == 3
    traffic = alg_per_launch * ((445.7 if cw8 else 618.5) / 7961.2)
    layout_name = {0: "binary DFS", 1: "binary BFS", 2: "4-wide", 3: "compressed 8-wide"}.get(
        (tuned or {}).get("node_order", 0), "binary DFS")

    cpu_baseline = builder = None
    if rank == 0 and world == 1:
        cpu_baseline = cpu_baseline_run(scenes, args.cpu_sample_s)
        if args.cpu_sample_s > 0:
            builder = build_baseline(scenes)

    # ---- config 5: served jobs (continuous batching) vs plain one-at-a-time launches.
    serving = None
    if args.serve_jobs > 0:
        del batch
        batch = None
        from renderbox2_b200.workloads import serving as serving_run
        serving = serving_run(n_jobs=args.serve_jobs)

    value = batch_rate / 1e6
    plain_value = plain_rate / 1e6
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(batch_total / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded PCG32 scenes and rays)",
        "config": {
            "workload": "config 4: 64 heightfield scenes, log-uniform 1k..2M triangles, 1M incoherent "
                        "diffuse-bounce rays per scene, 50% closest-hit / 50% any-hit (occlusion)",
            "mode": "batched: one persistent graph-replayed launch over 128 jobs (autotuned)",
            "autotuned": tuned, "scenes": len(scenes), "triangles": int(sum(s["tris"] for s in scenes)),
            "rays_per_step": int(total_rays), "l2": "flushed (256 MB write) between timed steps",
            "bvh_device_bytes": int(bvh_bytes), "build_s_host": round(build_s, 2), "parallelism": "replicas",
        },
        "plain_launches_mrays": round(plain_value, 2),
        "batched_over_plain": round(value / plain_value, 3),
        "plain_closest_hit_mrays": round(world * n_ch_total * args.steps / (ch_ms.sum() / 1e3) / 1e6, 2),
        "plain_any_hit_mrays": round(world * (total_rays - n_ch_total) * args.steps / (ah_ms.sum() / 1e3) / 1e6, 2),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak, "unit": "GB/s",
                     "frac": round(achieved / hbm_peak, 4), "traffic": round(traffic),
                     "kernel": f"k_trace_jobs<BLOCK, REGS, LAYOUT> (batched, 1 launch/step, {layout_name} nodes)",
                     "peak_source": peak_src,
                     "alg_bytes_per_launch": round(alg_per_launch),
                     "alg_bytes_per_ray": round(alg_per_launch / total_rays, 1),
                     "traffic_source": "scaled from ncu dram bytes of the 8 x 500k-triangle batched capture"},
        "e2e": {"value": round(e2e_rate / 1e6, 2), "unit": "Mrays/s",
                "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": d2h_bytes,
                "path": f"rb2_trace_host_jobs over the 128 jobs (pinned host buffers, chunks of {args.e2e_chunk} "
                        f"rays through {args.e2e_depth} streams, copies in the timed region, CUDA events)",
                "single_call_mrays": round(e2e_single_rate / 1e6, 2),
                "single_call_path": "one blocking rb2_trace_host per job, 16-byte hits for every ray"},
        "gpu_launches": args.steps * (1 + 2 * len(scenes)),
        "gpu_launches_note": "timed region: batched steps (1 traversal launch each) + plain steps (2 per scene)",
        "clocks": clocks,
    }
    if cpu_baseline is not None:
        line["cpu_baseline"] = cpu_baseline
    if builder is not None:
        line["build_baseline"] = builder
    if serving is not None:
        line["serving"] = serving
    if rank == 0:
        print(json.dumps(line), flush=True)
    del batch
    torch.cuda.synchronize(dev)


def run_workload(args, rank, local_rank):
    """Configs 1-3 at full size (one JSON line, not the headline)."""
    import torch

    from renderbox2_b200.workloads import integrator
    torch.cuda.set_device(local_rank)
    keep = {}
    r = integrator(args.workload, keep=keep)
    if rank == 0:
        names = {"ao": "config 1: ambient occlusion", "pt": "config 2: wavefront path tracing",
                 "bdpt": "config 3: BDPT with light-vertex cache",
                 "raycast": "config-2 scene, camera and spp: ray casting (primary rays, primitive-id shading)"}
        line = {"metric": "samples/s and Mrays/s", "workload": names[args.workload], **r}
        if world_of_env() == 1:
            base, counts = integrator_cpu_baseline(args.workload, keep)
            if args.cpu_sample_s > 0:
                line["cpu_baseline"] = base
            if counts is not None:
                line["roofline"] = integrator_roofline(args.workload, r, counts)
        print(json.dumps(line), flush=True)


def world_of_env() -> int:
    return int(os.environ.get("WORLD_SIZE", "1"))


def integrator_cpu_baseline(kind, keep):
    """The FP64 CPU integrators (oracle) on all host cores over a sample of the
    same frame: config 1 at full size (all 512 x 512 pixels, 16 AO rays),
    configs 2 and 3 on a grid of 128 x 72 pixels spread over the whole frame at
    the configs' spp.  Also returns the oracle's canonical visit counts per
    ray type over that sample (for the trace-stage roofline)."""
    import oracle
    c, scene, bvh = keep["config"], keep["scene"], keep["bvh"]
    W, H = c["width"], c["height"]
    cores = os.cpu_count() or 1
    bufs = bvh.buffers_view()
    if not oracle.have_ref():
        return {"unavailable": "reference camera library not built"}, None
    oracle.counts_reset(True)
    if kind == "ao":
        ii, jj = np.meshgrid(np.arange(W), np.arange(H))
        xy = np.stack([ii.ravel() + 0.5, jj.ravel() + 0.5], 1).astype(np.float32)
        rays = oracle.ref_camera_rays(keep["eye"], keep["lookat"], c["up"], W, H, c["fov"], xy)
        t0 = time.perf_counter()
        oracle.ao(bufs, scene.vertices, scene.indices, rays, c["ao_samples"], c["ao_radius"], seed=c["ao_seed"])
        dt = time.perf_counter() - t0
        samples = xy.shape[0] * c["ao_samples"]
        crop = f"full frame {W}x{H}, {c['ao_samples']} AO rays per pixel"
    elif kind == "raycast":
        gx, gy = 128, 72
        sx, sy = W // gx, H // gy
        spp = c["spp"]
        ii, jj = np.meshgrid(np.arange(gx) * sx + sx // 2, np.arange(gy) * sy + sy // 2)
        rng = np.random.Generator(np.random.PCG64(5))
        base = np.stack([ii.ravel(), jj.ravel()], 1)
        xy = (np.tile(base, (spp, 1)) + rng.uniform(0, 1, (base.shape[0] * spp, 2))).astype(np.float32)
        rays = oracle.ref_camera_rays(keep["eye"], keep["lookat"], c["up"], W, H, c["fov"], xy)
        nodes, woop, tri = bvh.get_node_buffer(), bvh.get_tri_woop_buffer(), bvh.get_tri_index_buffer()
        t0 = time.perf_counter()
        hits, cnt = oracle.trace(nodes, woop, tri, rays, counts=True)
        oracle.raycast_shade(hits["prim"], 0, scene.vertices, scene.indices, scene.material_ids, scene.albedo,
                             scene.emission)
        dt = time.perf_counter() - t0
        oracle.counts_reset(False)
        samples = base.shape[0] * spp
        crop = f"{gx}x{gy} pixels on a stride-{sx}x{sy} grid over the {W}x{H} frame at {spp} spp"
        counts = {"camera": {"rays": int(rays.shape[0]), "nodes": int(cnt["nodes"].sum()),
                             "tris": int(cnt["tris"].sum()), "leafterms": int(cnt["leafterms"].sum())}}
        return ({"value": round(samples / dt, 1), "unit": "samples/s", "cores": cores, "kind": "port",
                 "sample": f"{crop}: {samples:,} samples in {dt:.1f}s, CPU traversal (oracle) and ray-cast "
                           f"shading, OpenMP over {cores} threads"}, counts)
    else:
        gx, gy = 128, 72
        sx, sy = W // gx, H // gy
        spp = c["spp"]
        ii, jj = np.meshgrid(np.arange(gx) * sx + sx // 2, np.arange(gy) * sy + sy // 2)
        rng = np.random.Generator(np.random.PCG64(5))
        base = np.stack([ii.ravel(), jj.ravel()], 1)
        lights = np.asarray(scene.light_ids_to_primitive_ids, np.uint32)
        if kind == "pt":
            xy = (np.repeat(base, spp, axis=0) + rng.uniform(0, 1, (base.shape[0] * spp, 2))).astype(np.float32)
            rays = oracle.ref_camera_rays(keep["eye"], keep["lookat"], c["up"], W, H, c["fov"], xy)
            t0 = time.perf_counter()
            oracle.pt(bufs, scene.vertices, scene.indices, scene.material_ids, scene.albedo, scene.emission, lights,
                      rays, c["max_depth"], c["rr_start"], c["rr_prob"], seed=3)
            dt = time.perf_counter() - t0
        else:
            xy = (np.tile(base, (spp, 1)) + rng.uniform(0, 1, (base.shape[0] * spp, 2))).astype(np.float32)
            rays = oracle.ref_camera_rays(keep["eye"], keep["lookat"], c["up"], W, H, c["fov"], xy)
            t0 = time.perf_counter()
            oracle.bdpt(bufs, scene.vertices, scene.indices, scene.material_ids, scene.albedo, scene.emission, lights,
                        rays, base.shape[0], spp, base.shape[0], c["max_path_length"], c["lvc_connections"], 3, 0.95,
                        seed=3)
            dt = time.perf_counter() - t0
        samples = base.shape[0] * spp
        crop = f"{gx}x{gy} pixels on a stride-{sx}x{sy} grid over the {W}x{H} frame at {spp} spp"
    counts = oracle.counts_read()
    oracle.counts_reset(False)
    return ({"value": round(samples / dt, 1), "unit": "samples/s", "cores": cores, "kind": "port",
             "sample": f"{crop}: {samples:,} samples in {dt:.1f}s, FP64 CPU integrator (oracle), "
                       f"OpenMP over {cores} threads"}, counts)


def integrator_roofline(kind, r, counts):
    """Trace-stage roofline of configs 1-3: algorithmic bytes of the frame's
    rays (GPU ray counts per type x the oracle's mean bytes per ray of that
    type, from its own rays of the same distributions) / the GPU time of the
    traversal launches (CUDA events around each)."""
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    out_b = {"camera": 16, "extension": 16, "light": 16, "shadow": 1, "connection": 1}

    def bpr(t):
        c = counts[t]
        if not c["rays"]:
            return 0.0
        return 32 + (64 * c["nodes"] + 48 * c["tris"] + 16 * c["leafterms"]) / c["rays"] + out_b[t]

    st = r["stats"]
    if kind == "ao":
        npix = r["width"] * r["height"]
        hit_frac = counts["shadow"]["rays"] / max(1, counts["camera"]["rays"] * (r["samples"] // npix))
        gpu = {"camera": npix, "shadow": r["samples"] * hit_frac}
    elif kind == "raycast":
        gpu = {"camera": st["primary_rays"]}
    else:
        gpu = {"camera": st["primary_rays"], "extension": st["extension_rays"], "shadow": st["shadow_rays"],
               "connection": st["connection_rays"], "light": st["light_rays"]}
    alg = sum(n * bpr(t) for t, n in gpu.items())
    trace_s = st["trace_ms"] / 1e3
    if trace_s <= 0:
        return None
    ach = alg / trace_s / 1e9
    return {"bound": "hbm", "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s", "frac": round(ach / hbm, 4),
            "traffic": None, "alg_bytes_per_frame": round(alg), "trace_ms": round(st["trace_ms"], 3),
            "bytes_per_ray": {t: round(bpr(t), 1) for t in gpu},
            "note": "peak = measured HBM copy; the BVHs of configs 1 and 2 fit the 126 MB L2, so the traversal "
                    "there is L2-bound and frac can exceed what HBM alone would allow"}


def cpu_baseline_run(scenes, budget_s: float):
    """Oracle traversal on all host cores over a bounded sample: equal share of
    each scene's closest-hit and any-hit rays, sized to ~budget_s seconds."""
    import oracle
    cores = os.cpu_count() or 1
    # Calibrate on a small sample, then size the measured sample to the budget.
    per = 512
    for _ in range(2):
        t0 = time.perf_counter()
        n = trace_sample(oracle, scenes, per)
        dt = time.perf_counter() - t0
        if dt > 0.5:
            break
        per *= 4
    rate = n / dt
    per = int(max(256, min(scenes[0]["rays"].shape[0] // 2, per * budget_s / max(dt, 1e-3))))
    t0 = time.perf_counter()
    n = trace_sample(oracle, scenes, per)
    dt = time.perf_counter() - t0
    return {"value": round(n / dt / 1e6, 3), "unit": "Mrays/s", "cores": cores, "kind": "port",
            "sample": f"{per} closest-hit + {per} any-hit rays from each of {len(scenes)} scenes "
                      f"({n:,} rays, {dt:.1f}s), oracle C restatement, OpenMP over {cores} threads"}


def build_baseline(scenes, budget_tris: int = 30_000):
    """SBVH build time: the reference's own host builder (compiled from its
    sources, single-threaded as written) against this library's builder on
    the same smallest config-4 scenes (about budget_tris triangles in all),
    with one thread and with all threads."""
    import oracle

    import renderbox2_b200 as rb
    if not oracle.have_ref():
        return {"unavailable": "reference builder library not built"}
    pick, tot = [], 0
    for s in sorted(scenes, key=lambda s: s["tris"]):
        if tot + s["tris"] > budget_tris and pick:
            break
        pick.append(s)
        tot += s["tris"]
    t0 = time.perf_counter()
    for s in pick:
        oracle.ref_build(s["scene"].vertices, s["scene"].indices)
    ref_s = time.perf_counter() - t0
    out = {"scenes": len(pick), "triangles": tot, "reference_s": round(ref_s, 3)}
    for threads, key in ((1, "rb2_1thread_s"), (0, "rb2_all_threads_s")):
        t0 = time.perf_counter()
        for s in pick:
            rb.BVH(s["scene"], params=rb.BuildParams(num_threads=threads))
        out[key] = round(time.perf_counter() - t0, 3)
    out["speedup_1thread"] = round(ref_s / max(out["rb2_1thread_s"], 1e-9), 1)
    out["speedup_all_threads"] = round(ref_s / max(out["rb2_all_threads_s"], 1e-9), 1)
    out["cores"] = os.cpu_count() or 1
    return out


def trace_sample(oracle, scenes, per):
    n = 0
    for s in scenes:
        nodes, woop, tri = s["bvh"].buffers_view()
        ch = s["rays"][: min(per, s["n_ch"])]
        ah = s["rays"][s["n_ch"]: s["n_ch"] + per]
        oracle.trace(nodes, woop, tri, ch, any_hit=False)
        oracle.trace(nodes, woop, tri, ah, any_hit=True)
        n += ch.shape[0] + ah.shape[0]
    return n


# ------------------------------------------------------------------- reference arm
def run_reference(args, rank, world):
    if rank != 0:
        return
    scenes, _ = build_workload(args.scenes, args.rays_per_scene)
    import oracle
    cores = os.cpu_count() or 1
    per = max(256, args.ref_rays_per_scene)
    for _ in range(args.warmup):
        trace_sample(oracle, scenes, min(per, 256))
    times, n = [], 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        n = trace_sample(oracle, scenes, per)
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = n * args.steps / tot / 1e6
    sample = (f"{per} closest-hit + {per} any-hit rays from each of {len(scenes)} scenes per step "
              f"({n:,} rays), CPU restatement of the reference traversal (the reference has no host "
              f"traversal), OpenMP over {cores} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(tot / args.steps * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "config 4: 64 heightfield scenes, log-uniform 1k..2M triangles, incoherent "
                               "diffuse-bounce rays, 50% closest-hit / 50% any-hit", "parallelism": "host cores"},
        "cpu_baseline": {"value": round(value, 3), "unit": "Mrays/s", "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------- dist glue
def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world, dev) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, local_ms: float, world: int, dev) -> tuple[float, float]:
    """Replicas: every rank processes units_per_rank in local_ms; the job's
    rate is all ranks' units over the slowest rank's time.  Returns
    (units per second, max-over-ranks ms)."""
    ms = max_over_ranks(float(local_ms), world, dev)
    return world * units_per_rank / (ms / 1e3), ms


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["rb2", "reference"], default="rb2")
    ap.add_argument("--scenes", type=int, default=64)
    ap.add_argument("--rays-per-scene", type=int, default=1 << 20)
    ap.add_argument("--ref-rays-per-scene", type=int, default=2048)
    ap.add_argument("--cpu-sample-s", type=float, default=15.0)
    ap.add_argument("--e2e-chunk", type=int, default=1 << 20, help="rays per chunk of the pipelined host path")
    ap.add_argument("--e2e-depth", type=int, default=4, help="streams of the pipelined host path")
    ap.add_argument("--serve-jobs", type=int, default=10000,
                    help="config-5 jobs in the serving measurement (0: skip)")
    ap.add_argument("--workload", choices=["trace", "ao", "pt", "bdpt", "raycast"], default="trace",
                    help="trace: the headline config-4 line; ao/pt/bdpt: configs 1-3 at full size")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if args.impl == "rb2":
            torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl" if args.impl == "rb2" else "gloo",
                                timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        elif args.workload != "trace":
            run_workload(args, rank, local_rank)
        else:
            run_rb2(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
