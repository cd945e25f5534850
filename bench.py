"""Benchmark: incoherent ray-query throughput on one B200 (config 4 workload).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl rb2|reference]
                  [--rays-per-scene R] [--scenes S]
                  [--workload trace|ao|pt|bdpt|raycast|profile|serve-curve]

One step = every scene's ray batch traced once: 64 heightfield scenes with
log-uniform 1k..2M triangles (built with the benchmark SAH costs,
configs.BUILD), 1M incoherent diffuse-bounce rays per scene, 50 % closest-hit
and 50 % any-hit (occlusion), in one batched launch whose configuration the
autotuner picks (node layout, launch shape, fetch and node-phase thresholds,
ray reordering; a reordering sort, when picked, runs inside the step).  Inputs are resident in HBM when the timed region
starts; L2 is flushed (256 MB write) between timed steps.  `e2e` repeats the step through the host-buffer C-ABI call
(rb2_trace_host_jobs: pinned host rays in, hits / occlusion bytes out, the
copies pipelined with traversal over several streams), copies included.
After timing, 4096 rays per scene and mode of the timed launch's outputs
(device and end-to-end) are checked against the CPU oracle on the same BVH
buffers; any mismatch makes the run exit non-zero.  The default line also
carries the configs 1-3 frame times (AO, path tracing, BDPT) and the serving
measurement (config 5).  Under torchrun each rank runs the same workload on
its own GPU (replicas, no collective); `value` = all ranks' rays /
max-over-ranks time.

--impl reference times the reference's own CPU path on the host cores: its
SBVH builder (compiled from the reference sources) builds the smaller scenes
of the same workload, and the CPU restatement of its traversal (the
reference has no host traversal) traces each scene's full ray batch.  That
process loads no part of this library.

--workload profile runs one batched launch configuration over a small case
repeatedly (for ncu captures; see --profile-* options); --node-threshold sets
the integrators' node-phase threshold in the ao/pt/bdpt/raycast lines;
--batch-config fixes
the headline's batch configuration instead of autotuning it (for repeatable
launch lists); --workload serve-curve measures config-5 latency against
offered load.
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
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mrays/s incoherent closest-hit; served-job p50/p99 vs plain launches, 1 B200"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ----------------------------------------------------------------------------- workload
def build_workload(n_scenes: int, rays_per_scene: int, seed_base: int = 4, tri_cost: float | None = None,
                   threads: int = 0):
    """The batching workload's scenes (config 4), built with the benchmark SAH
    costs (configs.BUILD; `tri_cost` overrides the triangle cost) on `threads`
    host threads (0: all)."""
    import renderbox2_b200 as rb
    from renderbox2_b200.accel import BuildParams, Platform
    from renderbox2_b200.configs import BUILD, CONFIG4, config4_triangle_counts
    platform = Platform(sah_node_cost=BUILD["sah_node_cost"],
                        sah_triangle_cost=BUILD["sah_triangle_cost"] if tri_cost is None else tri_cost)
    counts = config4_triangle_counts(dict(CONFIG4, n_scenes=64))[:n_scenes]
    scenes = []
    t0 = time.time()
    build_s = 0.0
    for k, tris in enumerate(counts):
        sc = rb.heightfield_for_triangles(seed=seed_base * 1000 + k, n_tris=tris)
        tb = time.time()
        bvh = rb.BVH(sc, platform=platform, params=BuildParams(num_threads=threads))
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


def sample_index(n: int, per: int) -> np.ndarray:
    """Evenly spread sample of `per` indices out of n (all when n <= per)."""
    return np.linspace(0, n - 1, min(per, n)).astype(np.int64) if n else np.zeros(0, np.int64)


def oracle_sample(scenes, per_scene: int, nthreads: int = 0):
    """The oracle on an evenly spread sample of each scene's closest-hit and
    any-hit rays: hit records (for the parity check of the timed launch) and
    canonical single-lane visit counts (for the algorithmic bytes).  Returns
    one dict per scene: mode -> {idx, hits, bytes_per_ray, nodes, tris}."""
    import oracle
    out = []
    for s in scenes:
        nodes, woop, tri = s["bvh"].buffers_view()
        res = {}
        for mode, sl in (("ch", slice(0, s["n_ch"])), ("ah", slice(s["n_ch"], None))):
            r = s["rays"][sl]
            idx = sample_index(r.shape[0], per_scene)
            hits, cnt = oracle.trace(nodes, woop, tri, r[idx], any_hit=(mode == "ah"), counts=True,
                                     nthreads=nthreads)
            out_b = 16 if mode == "ch" else 1
            bpr = 32 + 64 * cnt["nodes"].astype(np.float64) + 48 * cnt["tris"] + 16 * cnt["leafterms"] + out_b
            res[mode] = dict(idx=idx, hits=hits, bytes_per_ray=float(bpr.mean()) if idx.size else 0.0,
                             nodes=float(cnt["nodes"].mean()) if idx.size else 0.0,
                             tris=float(cnt["tris"].mean()) if idx.size else 0.0)
        out.append(res)
    return out


def parity_check(scenes, samples, got_ch, got_occ, count_ties: bool = True):
    """Closest hits: prim, t, u and v bits equal to the oracle's, except at a
    confirmed tie (both triangles accept the ray at the same t: the layouts
    that test triangles in another order may report the other one, the
    reference's rule being tmin < t < hitT, kepler_dynamic_fetch.h:264).
    Occlusion bytes equal to the oracle's any-hit decision.  `got_ch[k]` /
    `got_occ[k]`: the GPU's records at samples[k]["ch"/"ah"]["idx"].  Also
    counts the sampled closest-hit rays on which a tie exists (oracle, BVH
    walk)."""
    import oracle
    n = mism = divergent = ties = culled = 0
    first = None
    for k, (s, smp) in enumerate(zip(scenes, samples)):
        nodes, woop, tri = s["bvh"].buffers_view()
        want = smp["ch"]["hits"]
        got = np.asarray(got_ch[k])
        rays = s["rays"][: s["n_ch"]][smp["ch"]["idx"]]
        n += want.shape[0]
        if want.shape[0]:
            g = got.view(np.uint32)
            ok = (got[:, 0] == want["prim"]) & (g[:, 1] == want["t"].view(np.uint32)) & \
                (g[:, 2] == want["u"].view(np.uint32)) & (g[:, 3] == want["v"].view(np.uint32))
            bad = np.nonzero(~ok)[0]
            slots = oracle.woop_slots_of(woop, tri) if bad.size else {}
            for b in bad:
                if got[b, 0] != want["prim"][b] and g[b, 1] == want["t"].view(np.uint32)[b] and \
                        oracle.is_tie(woop, tri, slots, rays[b], got[b, 0], want["prim"][b]):
                    divergent += 1
                elif (rays[b, 4:7] == 0.0).any() and got[b].view(np.float32)[1] < want["t"][b] and \
                        oracle.bruteforce(woop, tri, rays[b:b + 1])["t"][0] == got[b].view(np.float32)[1]:
                    # A direction component exactly 0 along a box boundary plane: the
                    # reference's slab test culls that box; the widened 8-wide boxes do not.
                    culled += 1
                else:
                    mism += 1
                    if first is None:
                        first = {"scene": k, "mode": "closest", "ray": int(smp["ch"]["idx"][b]),
                                 "gpu": [int(x) for x in got[b]], "oracle_prim": int(want["prim"][b])}
            if count_ties:
                ties += int((oracle.tie_count(woop, tri, rays, want, nodes=nodes) >= 2).sum())
        want_o = smp["ah"]["hits"]["prim"] >= 0
        got_o = np.asarray(got_occ[k]).astype(bool)
        n += want_o.shape[0]
        bad_o = np.nonzero(got_o != want_o)[0]
        mism += int(bad_o.size)
        if bad_o.size and first is None:
            first = {"scene": k, "mode": "occlusion", "ray": int(smp["ah"]["idx"][bad_o[0]])}
    out = {"rays": int(n), "mismatches": int(mism), "ties": int(ties), "tie_divergent": int(divergent),
           "reference_culled": int(culled)}
    if first is not None:
        out["first_mismatch"] = first
    return out


# ------------------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = Path(tempfile.mkdtemp(prefix="rb2_clocks_")) / "clocks.csv"

    def __enter__(self):
        try:
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
# DRAM bytes per algorithmic byte of the batched traversal kernel, from ncu
# (dram__bytes_read.sum + dram__bytes_write.sum of one launch) on a case small
# enough for the profiler: the first 8 scenes of this workload (its triangle
# counts and seeds, 524,288 rays each, 7,023.9 MB of algorithmic bytes), block
# 256.  Keyed by (node order, ray reordering on): the compressed 8-wide kernel
# at 64 registers on rays in their own order with node-phase threshold 12
# (benchmark SAH costs, 6,944.2 MB algorithmic); the binary BFS kernel at 48
# registers on rays reordered at 5 bits per axis (reference costs, node-phase
# threshold 1); the compressed kernel at 64 registers on rays reordered at 4
# bits per axis (benchmark costs, node-phase threshold 1).
DRAM_PER_ALG_BYTE = {
    (3, False): (392.0e6 / 6944.2e6, "first 8 scenes of this workload, 4.19M rays, compressed 8-wide layout, "
                                     "node-phase threshold 12"),
    (1, True): (595.1e6 / 7023.9e6, "first 8 scenes of this workload, 4.19M rays, binary BFS layout, rays "
                                    "reordered"),
    (3, True): (423.9e6 / 6944.2e6, "first 8 scenes of this workload, 4.19M rays, compressed 8-wide layout, "
                                    "rays reordered"),
}


def l2_copy_gbs(dev, stream, mbytes: int = 32, reps: int = 200) -> float:
    """Achieved L2 bandwidth: a device-to-device copy of an `mbytes` MB
    buffer into another (both resident in the 126 MB L2 after the first
    pass), repeated; read + write bytes over CUDA-event time, best of 3."""
    import torch
    n = mbytes * 1024 * 1024 // 4
    a = torch.ones(n, dtype=torch.float32, device=dev)
    b = torch.empty_like(a)
    best = 0.0
    with torch.cuda.stream(stream):
        for _ in range(3):
            for _ in range(5):
                b.copy_(a)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                b.copy_(a)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            best = max(best, 2.0 * a.numel() * 4 * reps / (e0.elapsed_time(e1) / 1e3) / 1e9)
    del a, b
    return best


def run_rb2(args, rank, world, local_rank):
    import torch

    import renderbox2_b200 as rb
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    # Ranks on one host share its cores for the builds.
    threads = max(1, (os.cpu_count() or 1) // world) if world > 1 else 0
    scenes, build_s = build_workload(args.scenes, args.rays_per_scene, tri_cost=args.sah_triangle_cost,
                                     threads=threads)
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
    # Parity sample: the same evenly spread rays the oracle traces below.
    idx_ch = [torch.from_numpy(sample_index(s["n_ch"], args.parity_rays)).to(dev) for s in scenes]
    idx_ah = [torch.from_numpy(sample_index(s["rays"].shape[0] - s["n_ch"], args.parity_rays)).to(dev)
              for s in scenes]

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
    jobs, ch_jobs = [], []
    for k, s in enumerate(scenes):
        jobs.append((tracers[k], d_rays[k][: s["n_ch"]], rb.MODE_CLOSEST, d_hits[k], None))
        jobs.append((tracers[k], d_rays[k][s["n_ch"]:], rb.MODE_OCCLUSION, d_occ[k], None))
        ch_jobs.append(jobs[-2])
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

    def plain_timed():
        ch_ms, ah_ms = np.zeros(len(scenes)), np.zeros(len(scenes))

        def collect():
            for k in range(len(scenes)):
                ch_ms[k] += pev[k][0][0].elapsed_time(pev[k][0][1])
                ah_ms[k] += pev[k][1][0].elapsed_time(pev[k][1][1])

        for _ in range(args.warmup):
            plain_step(False)
        torch.cuda.synchronize(dev)
        barrier(world)
        ms = timed(lambda: plain_step(True), args.steps, collect)
        return ms, ch_ms, ah_ms

    def gather_outputs():
        return ([d_hits[k][idx_ch[k]].cpu().numpy() for k in range(len(scenes))],
                [d_occ[k][idx_ah[k]].cpu().numpy() for k in range(len(scenes))])

    # The plain path is timed first, with the tracers' defaults (the reference's
    # DFS Compact2 layout, default launch shape), before the autotuner changes
    # any tracer's layout; then the batched launch is tuned (untimed), captured
    # and timed; then a batch of the closest-hit jobs alone; then the plain
    # path again with the autotuned layout and launch shape, which separates
    # the gain of batching from the gain of the layout.  Clocks are sampled
    # across all timed regions.
    with ClockSampler(local_rank) as clk:
        plain_ms, ch_ms, ah_ms = plain_timed()
        if args.batch_config:
            batch.set_config(**json.loads(args.batch_config))
            tuned, tuned_ms = batch.config(), None
        else:
            tuned, tuned_ms = batch.autotune(stream=stream, reps=5)
        batch.capture(stream)
        for _ in range(args.warmup):
            batch.launch(stream)
        torch.cuda.synchronize(dev)
        barrier(world)
        batch_ms = timed(lambda: batch.launch(stream), args.steps)
        got_ch, got_occ = gather_outputs()  # outputs of the last timed launch
        batch_status = batch.status(stream)
        # The same launch without ray reordering (the plain launches have none).
        unsorted_ms = None
        if tuned.get("reorder", 0):
            batch.set_config(**dict(tuned, reorder=0))
            batch.capture(stream)
            for _ in range(args.warmup):
                batch.launch(stream)
            torch.cuda.synchronize(dev)
            barrier(world)
            unsorted_ms = timed(lambda: batch.launch(stream), args.steps)
            batch_status |= batch.status(stream)
            batch.set_config(**tuned)
        ch_batch = rb.TraceBatch(ch_jobs)
        ch_batch.set_config(**tuned)
        ch_batch.capture(stream)
        for _ in range(args.warmup):
            ch_batch.launch(stream)
        torch.cuda.synchronize(dev)
        barrier(world)
        ch_batch_ms = timed(lambda: ch_batch.launch(stream), args.steps)
        ch_batch_status = ch_batch.status(stream)
        for t in tracers:  # the batch already switched every tracer to the tuned layout
            t.set_launch(ctas_per_sm=tuned["ctas_per_sm"], fetch_threshold=tuned["fetch_threshold"],
                         block_threads=tuned["block_threads"], regs=tuned["regs"])
        same_ms, same_ch_ms, same_ah_ms = plain_timed()
    clocks = clk.summary()
    plain_rate, _ = whole_job_rate(total_rays * args.steps, sum(plain_ms), world, dev)
    batch_rate, batch_total = whole_job_rate(total_rays * args.steps, sum(batch_ms), world, dev)
    ch_batch_rate, _ = whole_job_rate(n_ch_total * args.steps, sum(ch_batch_ms), world, dev)
    same_rate, _ = whole_job_rate(total_rays * args.steps, sum(same_ms), world, dev)
    unsorted_rate = (whole_job_rate(total_rays * args.steps, sum(unsorted_ms), world, dev)[0]
                     if unsorted_ms is not None else None)
    for t in tracers:
        assert t.status() == 0, "device status word set"
    assert batch_status == 0 and ch_batch_status == 0, "batch status word set"
    del ch_batch

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
    e2e_ch = [h_hits[k].numpy()[sample_index(s["n_ch"], args.parity_rays)] for k, s in enumerate(scenes)]
    e2e_occ = [h_occ[k].numpy()[sample_index(s["rays"].shape[0] - s["n_ch"], args.parity_rays)]
               for k, s in enumerate(scenes)]
    e2e_single_rate, _ = whole_job_rate(total_rays * e2e_single_steps, device_ms(e2e_single_step, e2e_single_steps),
                                        world, dev)
    l2_gbs = l2_copy_gbs(dev, stream)

    # ---- parity of the timed launch and of the end-to-end outputs against the oracle.
    samples = oracle_sample(scenes, args.parity_rays)
    parity = parity_check(scenes, samples, got_ch, got_occ)
    parity_e2e = parity_check(scenes, samples, e2e_ch, e2e_occ, count_ties=False)
    parity["e2e_mismatches"] = parity_e2e["mismatches"]
    parity["e2e_tie_divergent"] = parity_e2e["tie_divergent"]
    parity["checked"] = (f"{args.parity_rays} closest-hit + {args.parity_rays} any-hit rays per scene, evenly "
                         "spread: the last timed batched launch and the e2e host outputs against the CPU oracle "
                         "on the same BVH buffers (prim/t/u/v bits; occlusion bytes); ties = sampled closest-hit "
                         "rays that 2+ triangles accept at the same t")

    # ---- roofline: dominant kernel = the batched traversal launch (one per step).
    ch_bytes = sum(sm["ch"]["bytes_per_ray"] * s["n_ch"] for sm, s in zip(samples, scenes))
    ah_bytes = sum(sm["ah"]["bytes_per_ray"] * (s["rays"].shape[0] - s["n_ch"]) for sm, s in zip(samples, scenes))
    node_visits = sum(sm["ch"]["nodes"] * s["n_ch"] + sm["ah"]["nodes"] * (s["rays"].shape[0] - s["n_ch"])
                      for sm, s in zip(samples, scenes))
    tri_tests = sum(sm["ch"]["tris"] * s["n_ch"] + sm["ah"]["tris"] * (s["rays"].shape[0] - s["n_ch"])
                    for sm, s in zip(samples, scenes))
    launch_s = batch_total / 1e3 / args.steps
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "MEASURED_PEAKS.json hbm_gbs (measured)" if "hbm_gbs" in peaks else "fallback 6650 GB/s"
    alg_per_launch = ch_bytes + ah_bytes
    achieved = alg_per_launch / launch_s / 1e9
    order = (tuned or {}).get("node_order", 0)
    sorted_rays = bool((tuned or {}).get("reorder", 0))
    key = (order, sorted_rays)
    if key not in DRAM_PER_ALG_BYTE:  # the capture of the nearest variant: same ray order, binary or compressed
        key = (3, False) if order == 3 or not sorted_rays else (1, True)
    ratio, ratio_src = DRAM_PER_ALG_BYTE[key]
    traffic = alg_per_launch * ratio
    layout_name = {0: "binary DFS", 1: "binary BFS", 2: "4-wide", 3: "compressed 8-wide"}.get(order, "binary DFS")
    # kernels of the ray-reordering sort per batched launch: one pass (count, columns, 3 scan, scatter) at
    # 3-4 bits per axis, two passes at 5-6
    reorder_bits = (tuned or {}).get("reorder", 0)
    sort_launches = 0 if not reorder_bits else (6 if reorder_bits <= 4 else 12)

    cpu_baseline = builder = None
    if rank == 0 and world == 1:
        cpu_baseline = cpu_baseline_run(scenes, args.cpu_sample_s, args.ref_max_tris, args.ref_budget_tris)
        if args.cpu_sample_s > 0:
            builder = build_baseline(scenes)

    # ---- config 5: served jobs (continuous batching) vs plain one-at-a-time launches.
    serving = None
    del batch
    batch = None
    # Serving and configs 1-3 are one-GPU measurements: under torchrun only
    # rank 0 runs them (its line reports them), so N ranks do not pin N times
    # the serving buffers on the host.
    if args.serve_jobs > 0 and rank == 0:
        from renderbox2_b200.workloads import serving as serving_run
        serving = serving_run(n_jobs=args.serve_jobs, slots=args.serve_slots)

    # ---- configs 1-3: one frame each at full size (trace-stage roofline vs L2 or HBM).
    integrators = {}
    if args.integrators and rank == 0:
        for kind in ("ao", "pt", "bdpt"):
            integrators[kind] = integrator_summary(kind, l2_gbs, with_cpu=(rank == 0 and world == 1),
                                                   tri_cost=args.sah_triangle_cost)

    value = batch_rate / 1e6
    plain_value = plain_rate / 1e6
    same_value = same_rate / 1e6
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(batch_total / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded PCG32 scenes and rays)",
        "config": {
            "workload": "config 4: 64 heightfield scenes, log-uniform 1k..2M triangles, 1M incoherent "
                        "diffuse-bounce rays per scene, 50% closest-hit / 50% any-hit (occlusion)",
            "mode": "batched: one persistent graph-replayed launch over 128 jobs "
                    + ("(configuration given on the command line)" if args.batch_config else "(autotuned)"),
            "autotuned": tuned, "scenes": len(scenes), "triangles": int(sum(s["tris"] for s in scenes)),
            "rays_per_step": int(total_rays), "l2": "flushed (256 MB write) between timed steps",
            "bvh_device_bytes": int(bvh_bytes), "build_s_host": round(build_s, 2), "parallelism": "replicas",
            "bvh_build": {"sah_node_cost": _load_configs().BUILD["sah_node_cost"],
                          "sah_triangle_cost": (args.sah_triangle_cost if args.sah_triangle_cost is not None
                                                else _load_configs().BUILD["sah_triangle_cost"]),
                          "note": "this library's SBVH builder; the reference's Platform costs are 1 and 1"},
        },
        "parity": parity,
        "plain_launches_mrays": round(plain_value, 2),
        "batched_over_plain": round(value / plain_value, 3),
        "plain_closest_hit_mrays": round(world * n_ch_total * args.steps / (ch_ms.sum() / 1e3) / 1e6, 2),
        "plain_any_hit_mrays": round(world * (total_rays - n_ch_total) * args.steps / (ah_ms.sum() / 1e3) / 1e6, 2),
        "plain_same_layout_mrays": round(same_value, 2),
        "plain_same_layout_closest_hit_mrays": round(world * n_ch_total * args.steps / (same_ch_ms.sum() / 1e3) / 1e6,
                                                     2),
        "batched_over_plain_same_layout": round(value / same_value, 3),
        "batched_closest_hit_mrays": round(ch_batch_rate / 1e6, 2),
        "batched_closest_hit_over_plain_same_layout": round(
            ch_batch_rate / 1e6 / (world * n_ch_total * args.steps / (same_ch_ms.sum() / 1e3) / 1e6), 3),
        "batched_without_reorder_mrays": round(unsorted_rate / 1e6, 2) if unsorted_rate else None,
        "plain_note": "plain = 2 launches per scene (closest-hit half, any-hit half); default = the reference's DFS "
                      "layout and the default launch shape; same_layout = the autotuned layout and launch shape "
                      "(plain launches have no ray reordering; batched_without_reorder = the batched launch with "
                      "the tuned shape and reordering off)",
        "roofline": {"bound": "l2", "achieved": round(achieved, 1), "peak": round(l2_gbs, 1), "unit": "GB/s",
                     "frac": round(achieved / l2_gbs, 4), "traffic": round(traffic),
                     "kernel": f"k_trace_jobs<BLOCK, REGS, LAYOUT> (batched, 1 launch/step, {layout_name} nodes)"
                               + (f"; the step time includes the {sort_launches} ray-reordering launches before it"
                                  if sort_launches else ""),
                     "peak_source": "L2 copy bandwidth measured in this run (a 32 MB buffer copied repeatedly, "
                                    "CUDA events)",
                     "bound_note": "DRAM serves about 6 % of the algorithmic bytes (traffic below; L1 and L2 hit "
                                   "the rest), so the L2 is the memory level those bytes are bound by; the "
                                   "kernel itself is issue-bound (ncu: ALU pipe and issue slots, not memory)",
                     "hbm_peak": hbm_peak, "hbm_peak_source": peak_src,
                     "alg_frac_of_hbm": round(achieved / hbm_peak, 4),
                     "alg_bytes_per_launch": round(alg_per_launch),
                     "alg_bytes_per_ray": round(alg_per_launch / total_rays, 1),
                     "traffic_source": f"ncu DRAM bytes per algorithmic byte of a capture ({ratio_src}) x this "
                                       "launch's algorithmic bytes",
                     "dram_gbs": round(traffic / launch_s / 1e9, 1),
                     "dram_frac": round(traffic / launch_s / 1e9 / hbm_peak, 4),
                     "node_visits_per_s": round(node_visits / launch_s, 0),
                     "box_tests_per_s": round(2 * node_visits / launch_s, 0),
                     "tri_tests_per_s": round(tri_tests / launch_s, 0),
                     "tests_note": "canonical single-lane counts of the oracle on the binary tree (inner-node "
                                   "fetches, 2 box tests each; Woop triangle tests), per second of the batched "
                                   "launch"},
        "e2e": {"value": round(e2e_rate / 1e6, 2), "unit": "Mrays/s",
                "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": d2h_bytes,
                "path": f"rb2_trace_host_jobs over the 128 jobs (pinned host buffers, chunks of {args.e2e_chunk} "
                        f"rays through {args.e2e_depth} streams, copies in the timed region, CUDA events)",
                "single_call_mrays": round(e2e_single_rate / 1e6, 2),
                "single_call_path": "one blocking rb2_trace_host per job, 16-byte hits for every ray"},
        "gpu_launches": args.steps * (2 * (1 + sort_launches) + (1 if sort_launches else 0) + 4 * len(scenes)),
        "gpu_launches_note": f"timed region: batched steps (1 traversal launch each, after {sort_launches} "
                             "ray-reordering launches), closest-hit batch steps (the same), batched steps without "
                             "reordering (1 each, when reordering is on), plain steps with default and with tuned "
                             "layout (2 per scene each)",
        "clocks": clocks,
    }
    if cpu_baseline is not None:
        line["cpu_baseline"] = cpu_baseline
    if builder is not None:
        line["build_baseline"] = builder
    if serving is not None:
        line["serving"] = serving
    if integrators:
        line["integrators"] = integrators
    if rank == 0:
        print(json.dumps(line), flush=True)
    torch.cuda.synchronize(dev)
    if parity["mismatches"] or parity["e2e_mismatches"]:
        log(f"PARITY FAILURE: {parity}")
        sys.exit(3)


def integrator_summary(kind, l2_gbs, with_cpu=True, tri_cost=None):
    """One full-size frame of config 1 (AO), 2 (PT) or 3 (BDPT): frame time,
    samples/s, Mrays/s, the trace stage's roofline (against the L2 copy
    bandwidth measured in the run) and the FP64 CPU integrator on a small
    sample of the same frame."""
    from renderbox2_b200.workloads import integrator
    keep = {}
    r = integrator(kind, keep=keep, tri_cost=tri_cost)
    c = keep["bvh"].counts()
    bvh_bytes = int(c.n_nodes_u4 * 16 + c.n_woop_u4 * 16 + c.n_triidx * 4)
    out = {"ms_per_frame": r["ms"], "samples_per_s": r["samples_per_s"], "mrays_per_s": r["mrays_per_s"],
           "triangles": r["triangles"], "resolution": [r["width"], r["height"]], "node_order": r["node_order"],
           "binary_bvh_bytes": bvh_bytes}
    base, counts = integrator_cpu_baseline(kind, keep)
    if with_cpu:
        out["cpu_baseline"] = base
    if counts is not None:
        out["roofline"] = integrator_roofline(kind, r, counts, l2_gbs, "L2 copy bandwidth measured in this run")
    return out


def run_workload(args, rank, local_rank):
    """Configs 1-3 at full size (one JSON line, not the headline)."""
    import torch

    from renderbox2_b200.workloads import integrator
    torch.cuda.set_device(local_rank)
    keep = {}
    r = integrator(args.workload, keep=keep, tri_cost=args.sah_triangle_cost, node_threshold=args.node_threshold)
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
                dev = torch.device("cuda", local_rank)
                peak = l2_copy_gbs(dev, torch.cuda.Stream(device=dev))
                line["roofline"] = integrator_roofline(args.workload, r, counts, peak,
                                                       "L2 copy bandwidth measured in this run")
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


def _hbm_peak():
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    if "hbm_gbs" in peaks:
        return peaks["hbm_gbs"], "MEASURED_PEAKS.json hbm_gbs (measured)"
    return 6650.0, "fallback 6650 GB/s"


def integrator_roofline(kind, r, counts, peak, peak_src):
    """Trace-stage roofline of configs 1-3: algorithmic bytes of the frame's
    rays (GPU ray counts per type x the oracle's mean bytes per ray of that
    type, from its own rays of the same distributions) / the GPU time of the
    traversal launches (CUDA events around each), against `peak`: the L2
    copy bandwidth measured in the run, since L1 and L2 serve nearly all of a
    traversal's algorithmic bytes (ncu on the batching workload, whose BVHs
    are 21x the L2: DRAM moves about 6 % of them); the fraction of HBM is
    reported beside it."""
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
    hbm, _ = _hbm_peak()
    out = {"bound": "l2", "achieved": round(ach, 1), "peak": round(peak, 1),
           "unit": "GB/s", "frac": round(ach / peak, 4), "peak_source": peak_src, "traffic": None,
           "alg_frac_of_hbm": round(ach / hbm, 4),
           "alg_bytes_per_frame": round(alg), "trace_ms": round(st["trace_ms"], 3),
           "bytes_per_ray": {t: round(bpr(t), 1) for t in gpu}}
    if kind == "raycast":
        out["note"] = ("coherent camera rays: neighbouring lanes fetch the same nodes, which the L1 serves, so the "
                       "fraction can exceed 1; neither L2 nor HBM bounds this trace")
    elif kind == "pt":
        out["note"] = ("camera and extension rays leave neighbouring pixels' points in pixel order, so the L1 serves "
                       "part of the node fetches and the fraction of the L2 copy can exceed 1")
    return out


def host_cpu_model() -> str:
    """The host CPU's model name (/proc/cpuinfo), for the CPU legs' records."""
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline_run(scenes, budget_s: float, ref_max_tris: int, ref_budget_tris: int):
    """Oracle traversal on all host cores over a bounded sample: equal share of
    each scene's closest-hit and any-hit rays, sized to ~budget_s seconds.
    Also times the oracle over this library's trees for the scene subset the
    reference arm builds with the reference's builder (its full rays), so the
    two CPU figures can be compared on the same scenes and rays."""
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
    per = int(max(256, min(scenes[0]["rays"].shape[0] // 2, per * budget_s / max(dt, 1e-3))))
    t0 = time.perf_counter()
    n = trace_sample(oracle, scenes, per)
    dt = time.perf_counter() - t0
    out = {"value": round(n / dt / 1e6, 3), "unit": "Mrays/s", "cores": cores, "kind": "port",
           "cpu": host_cpu_model(),
           "sample": f"{per} closest-hit + {per} any-hit rays from each of {len(scenes)} scenes "
                     f"({n:,} rays, {dt:.1f}s), oracle C restatement, OpenMP over {cores} threads"}
    if budget_s > 0:
        # One thread on a sample sized to about a tenth of the budget (assuming
        # the all-core rate divides evenly over the cores).
        per1 = int(n / dt / cores * budget_s / 10 / (2 * len(scenes)))
        per1 = max(64, min(per1, per))
        t0 = time.perf_counter()
        n1 = trace_sample(oracle, scenes, per1, nthreads=1)
        dt1 = time.perf_counter() - t0
        out["single_thread"] = {"value": round(n1 / dt1 / 1e6, 3), "unit": "Mrays/s",
                                "sample": f"{per1} closest-hit + {per1} any-hit rays from each scene ({n1:,} rays, "
                                          f"{dt1:.1f}s), one thread"}
    sub = reference_subset([s["tris"] for s in scenes], ref_max_tris, ref_budget_tris)
    if sub and budget_s > 0:
        t0 = time.perf_counter()
        n = trace_sample(oracle, [scenes[k] for k in sub], 1 << 40)
        dt = time.perf_counter() - t0
        out["reference_subset"] = {"value": round(n / dt / 1e6, 3), "scenes": len(sub),
                                   "triangles": int(sum(scenes[k]["tris"] for k in sub)), "rays": n,
                                   "note": "the oracle over this library's trees of the scenes the reference arm "
                                           "builds with the reference builder, every ray of each"}
    return out


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


def trace_sample(oracle, scenes, per, nthreads: int = 0):
    """The oracle over `per` closest-hit and `per` any-hit rays of each scene
    (nthreads 0: all host threads); returns the rays traced."""
    n = 0
    for s in scenes:
        nodes, woop, tri = s["bvh"].buffers_view()
        ch = s["rays"][: min(per, s["n_ch"])]
        ah = s["rays"][s["n_ch"]: s["n_ch"] + per]
        oracle.trace(nodes, woop, tri, ch, any_hit=False, nthreads=nthreads)
        oracle.trace(nodes, woop, tri, ah, any_hit=True, nthreads=nthreads)
        n += ch.shape[0] + ah.shape[0]
    return n


# ------------------------------------------------------------------- reference arm
def _load_configs():
    """renderbox2_b200/configs.py loaded by file path, so the reference
    process never imports the package (nor loads its library)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_rb2_configs", ROOT / "renderbox2_b200" / "configs.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def reference_subset(tris, max_tris: int, budget_tris: int) -> list[int]:
    """Scenes the reference's single-threaded builder can build within the
    run: smallest first, each at most max_tris triangles, budget_tris in all.
    Returns scene indices in workload order."""
    pick, tot = [], 0
    for k in sorted(range(len(tris)), key=lambda k: tris[k]):
        if tris[k] > max_tris or tot + tris[k] > budget_tris:
            break
        pick.append(k)
        tot += tris[k]
    return sorted(pick)


def _ref_build_worker(item):
    """One scene through the reference's SBVH builder + Compact2 packer
    (compiled from its sources), in a worker process."""
    k, v, i = item
    import oracle
    t0 = time.perf_counter()
    r = oracle.ref_build(v, i)
    return k, r["nodes"], r["woop"], r["triidx"], time.perf_counter() - t0


def run_reference(args, rank, world):
    """The reference's CPU path on the host cores: the scenes of the batching
    workload that its builder can build in the run (reference_subset), built
    by that builder (one process per scene, all cores), then every ray of
    each built scene (the workload's 1M rays: closest-hit half and any-hit
    half, one call each) traced by the CPU restatement of its traversal on
    all cores.  Scenes and rays come from the oracle's copy of the workload
    generator; no part of this library is loaded."""
    if rank != 0:
        return
    import concurrent.futures as cf
    import multiprocessing as mp

    import oracle
    cores = os.cpu_count() or 1
    if not oracle.have_ref():
        print(json.dumps({"impl": "reference", "unavailable": "reference builder (oracle/_ref) not built"}),
              flush=True)
        return
    cfgs = _load_configs()
    c4 = cfgs.CONFIG4
    counts = cfgs.config4_triangle_counts(dict(c4, n_scenes=64))[: args.scenes]
    sub = reference_subset(counts, args.ref_max_tris, args.ref_budget_tris)
    t0 = time.time()
    scenes = []
    for k in sub:
        v, i = oracle.gen_heightfield_for_triangles(4000 + k, counts[k])
        rays, flags = oracle.gen_surface_rays(v, i, 4500 + k, args.rays_per_scene, c4["offset_scale"],
                                              c4["anyhit_fraction"])
        order = np.argsort(flags, kind="stable")
        scenes.append(dict(k=k, v=v, i=i, rays=np.ascontiguousarray(rays[order]), n_ch=int((flags == 0).sum()),
                           tris=int(i.shape[0])))
    gen_s = time.time() - t0
    t0 = time.time()
    work = sorted(range(len(scenes)), key=lambda j: -scenes[j]["tris"])
    build_cpu = 0.0
    with cf.ProcessPoolExecutor(max_workers=cores, mp_context=mp.get_context("spawn")) as ex:
        for j, nodes, woop, tri, dt in ex.map(_ref_build_worker, [(j, scenes[j]["v"], scenes[j]["i"]) for j in work]):
            scenes[j].update(nodes=nodes, woop=woop, tri=tri)
            build_cpu += dt
    build_wall = time.time() - t0
    log(f"reference arm: {len(scenes)} scenes, {sum(s['tris'] for s in scenes):,} triangles; generation "
        f"{gen_s:.1f}s, reference SBVH build {build_wall:.1f}s wall ({build_cpu:.1f}s over {cores} processes)")

    def step():
        n = 0
        for s in scenes:
            ch, ah = s["rays"][: s["n_ch"]], s["rays"][s["n_ch"]:]
            oracle.trace(s["nodes"], s["woop"], s["tri"], ch, any_hit=False)
            oracle.trace(s["nodes"], s["woop"], s["tri"], ah, any_hit=True)
            n += ch.shape[0] + ah.shape[0]
        return n

    for _ in range(args.warmup):
        step()
    times, n = [], 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        n = step()
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = n * args.steps / tot / 1e6
    tris = sum(s["tris"] for s in scenes)
    sample = (f"{len(scenes)} of the {len(counts)} scenes ({tris:,} triangles; every scene of at most "
              f"{args.ref_max_tris:,} triangles, {args.ref_budget_tris:,} in all) built by the reference SBVH "
              f"builder; all {args.rays_per_scene:,} rays of each per step ({n:,} rays), traced by the CPU "
              f"restatement of the reference traversal (the reference has no host traversal), OpenMP over "
              f"{cores} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(tot / args.steps * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "config 4: 64 heightfield scenes, log-uniform 1k..2M triangles, 1M incoherent "
                               "diffuse-bounce rays per scene, 50% closest-hit / 50% any-hit; the scenes the "
                               "reference builder builds within the run", "parallelism": "host cores",
                   "scenes": len(scenes), "triangles": tris, "rays_per_step": n},
        "cpu_baseline": {"value": round(value, 3), "unit": "Mrays/s", "cores": cores, "kind": "reference",
                         "cpu": host_cpu_model(), "sample": sample},
        "build": {"reference_sbvh_wall_s": round(build_wall, 2), "reference_sbvh_cpu_s": round(build_cpu, 2),
                  "processes": cores, "triangles": tris},
        "e2e": {"value": round(value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------- profile case
def run_profile(args, local_rank):
    """A small, repeatable case of the batched traversal for ncu captures:
    either the first --scenes scenes of the batching workload (its triangle
    counts and seeds) with --rays-per-scene rays each, or (with
    --profile-equal-tris T) --scenes heightfields of T/scenes triangles each
    (seeds 300+k, rays 400+k); half closest-hit / half occlusion jobs; one
    launch configuration; --launches launches, CUDA-event timed.  Prints the
    launch times and the algorithmic bytes per launch (oracle visit counts)."""
    import torch

    import renderbox2_b200 as rb
    torch.cuda.set_device(local_rank)
    if args.profile_equal_tris:
        per = max(1000, args.profile_equal_tris // args.scenes)
        scenes = []
        for k in range(args.scenes):
            sc = rb.heightfield_for_triangles(seed=300 + k, n_tris=per)
            rays, _ = rb.surface_rays(sc, seed=400 + k, n=args.rays_per_scene)
            scenes.append(dict(scene=sc, bvh=rb.BVH(sc), rays=rays, n_ch=args.rays_per_scene // 2,
                               tris=sc.num_triangles))
    else:
        scenes, _ = build_workload(args.scenes, args.rays_per_scene, tri_cost=args.sah_triangle_cost)
    keep, jobs = [], []
    for s in scenes:
        tr = rb.CudaTracer(s["bvh"])
        d = torch.from_numpy(s["rays"]).cuda()
        out_h = torch.empty((s["n_ch"], 4), dtype=torch.int32, device="cuda")
        out_o = torch.empty((s["rays"].shape[0] - s["n_ch"],), dtype=torch.uint8, device="cuda")
        jobs += [(tr, d[: s["n_ch"]], rb.MODE_CLOSEST, out_h, None), (tr, d[s["n_ch"]:], rb.MODE_OCCLUSION, out_o, None)]
        keep.append((tr, d, out_h, out_o))
    batch = rb.TraceBatch(jobs)
    batch.set_config(block_threads=args.profile_block, regs=args.profile_regs, node_order=args.profile_order,
                     fetch_threshold=args.profile_threshold, ctas_per_sm=args.profile_ctas, chunk=args.profile_chunk,
                     reorder=args.profile_reorder, node_threshold=args.profile_node_threshold)
    ms = []
    for _ in range(args.launches):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        batch.launch()
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    assert batch.status() == 0
    res = {"scenes": len(scenes), "triangles": int(sum(s["tris"] for s in scenes)),
           "rays": int(sum(s["rays"].shape[0] for s in scenes)), "launch_ms": ms, "config": batch.config()}
    if not args.no_oracle:
        smp = oracle_sample(scenes, args.parity_rays)
        alg = sum(sm["ch"]["bytes_per_ray"] * s["n_ch"] + sm["ah"]["bytes_per_ray"] * (s["rays"].shape[0] - s["n_ch"])
                  for sm, s in zip(smp, scenes))
        best = min(ms[1:] if len(ms) > 1 else ms)
        res.update(alg_bytes_per_launch=alg, achieved_gbs_best=alg / (best / 1e3) / 1e9)
    print(json.dumps(res), flush=True)


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
    ap.add_argument("--parity-rays", type=int, default=4096,
                    help="rays per scene and mode checked against the oracle after timing")
    ap.add_argument("--ref-max-tris", type=int, default=150_000,
                    help="reference arm: largest scene its builder builds")
    ap.add_argument("--ref-budget-tris", type=int, default=2_000_000,
                    help="reference arm: triangles built in all")
    ap.add_argument("--cpu-sample-s", type=float, default=15.0)
    ap.add_argument("--e2e-chunk", type=int, default=1 << 20, help="rays per chunk of the pipelined host path")
    ap.add_argument("--e2e-depth", type=int, default=4, help="streams of the pipelined host path")
    ap.add_argument("--serve-jobs", type=int, default=10000,
                    help="config-5 jobs in the serving measurement (0: skip)")
    ap.add_argument("--serve-slots", type=int, default=32, help="concurrent slots of the continuous server")
    ap.add_argument("--no-integrators", dest="integrators", action="store_false",
                    help="leave configs 1-3 out of the default line")
    ap.add_argument("--workload", choices=["trace", "ao", "pt", "bdpt", "raycast", "profile", "serve-curve"],
                    default="trace",
                    help="trace: the headline config-4 line; ao/pt/bdpt/raycast: one integrator config at full "
                         "size; profile: a small batched case for ncu; serve-curve: config-5 latency against "
                         "offered load")
    ap.add_argument("--launches", type=int, default=3, help="profile: launches")
    ap.add_argument("--no-oracle", action="store_true", help="profile: skip the algorithmic-byte count")
    ap.add_argument("--profile-equal-tris", type=int, default=0,
                    help="profile: equal heightfields of this many triangles in all instead of workload scenes")
    ap.add_argument("--profile-block", type=int, default=256)
    ap.add_argument("--profile-regs", type=int, default=64)
    ap.add_argument("--profile-order", type=int, default=3)
    ap.add_argument("--profile-threshold", type=int, default=28)
    ap.add_argument("--profile-node-threshold", type=int, default=0, help="profile: node-phase threshold (0: default)")
    ap.add_argument("--profile-ctas", type=int, default=0)
    ap.add_argument("--profile-chunk", type=int, default=1)
    ap.add_argument("--profile-reorder", type=int, default=0, help="profile: ray reordering bits per axis (0 off)")
    ap.add_argument("--sah-triangle-cost", type=float, default=None,
                    help="SAH triangle cost of the workloads' builds (configs 1-4; default: configs.BUILD; the "
                         "reference's is 1)")
    ap.add_argument("--node-threshold", type=int, default=0,
                    help="ao/pt/bdpt/raycast: the traversal's node-phase threshold (0: the layout's default)")
    ap.add_argument("--batch-config", default="",
                    help="trace: a JSON rb2_batch_config for the batched launch instead of the autotuner's pick "
                         "(for repeatable profiles)")
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
        elif args.workload == "profile":
            run_profile(args, local_rank)
        elif args.workload == "serve-curve":
            import torch

            from renderbox2_b200.workloads import serving_curve
            torch.cuda.set_device(local_rank)
            r = serving_curve(n_jobs=args.serve_jobs if args.serve_jobs != 10000 else 3000, slots=args.serve_slots)
            if rank == 0:
                print(json.dumps({"metric": "served-job latency against offered load (config 5)", **r}), flush=True)
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
