"""Small, self-contained traversal case for ncu captures and roofline bytes.

  python -m renderbox2_b200.profile_case [--tris 2000000] [--rays 1048576] [--mode ch|ah] [--launches 3]

One heightfield scene of --tris triangles (BVH larger than the 126 MB L2 at
the default size), --rays incoherent diffuse-bounce rays traced --launches
times with the persistent traversal kernel.  Prints the per-launch CUDA-event
time and the algorithmic bytes per launch from the oracle's canonical visit
counts (32 + 64*nodes + 48*tris + 16*terminators + output bytes per ray).
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--tris", type=int, default=2_000_000)
    ap.add_argument("--rays", type=int, default=1 << 20)
    ap.add_argument("--mode", choices=["ch", "ah"], default="ch")
    ap.add_argument("--launches", type=int, default=3)
    ap.add_argument("--no-oracle", action="store_true")
    ap.add_argument("--batched", type=int, default=0,
                    help="N > 0: N scenes of --tris/N triangles, half closest-hit / half occlusion jobs, one batched "
                         "launch per repetition with the given --block/--regs/--order")
    ap.add_argument("--block", type=int, default=256)
    ap.add_argument("--regs", type=int, default=64)
    ap.add_argument("--order", type=int, default=1)
    args = ap.parse_args()

    import torch

    import renderbox2_b200 as rb
    if args.batched > 0:
        return batched_case(args)
    scene = rb.heightfield_for_triangles(seed=77, n_tris=args.tris)
    bvh = rb.BVH(scene)
    rays, _ = rb.surface_rays(scene, seed=78, n=args.rays)
    tr = rb.CudaTracer(bvh)
    d = torch.from_numpy(rays).cuda()
    out_h = torch.empty((args.rays, 4), dtype=torch.int32, device="cuda")
    out_o = torch.empty((args.rays,), dtype=torch.uint8, device="cuda")
    ms = []
    for _ in range(args.launches):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        if args.mode == "ch":
            tr.trace(d, out=out_h)
        else:
            tr.trace_occlusion(d, out=out_o)
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    assert tr.status() == 0
    res = {"tris": scene.num_triangles, "rays": args.rays, "mode": args.mode, "bvh_bytes": tr.device_bytes(),
           "launch_ms": ms}
    if not args.no_oracle:
        import oracle
        nodes, woop, tri = bvh.buffers_view()
        idx = np.linspace(0, args.rays - 1, min(65536, args.rays)).astype(np.int64)
        _, cnt = oracle.trace(nodes, woop, tri, rays[idx], any_hit=args.mode == "ah", counts=True)
        out_b = 16 if args.mode == "ch" else 1
        bpr = 32 + 64 * cnt["nodes"].astype(np.float64) + 48 * cnt["tris"] + 16 * cnt["leafterms"] + out_b
        res.update(alg_bytes_per_ray=float(bpr.mean()), alg_bytes_per_launch=float(bpr.mean() * args.rays),
                   mean_nodes=float(cnt["nodes"].mean()), mean_tris=float(cnt["tris"].mean()),
                   mean_leafterms=float(cnt["leafterms"].mean()))
        best = min(ms[1:] if len(ms) > 1 else ms)
        res["achieved_gbs_best"] = res["alg_bytes_per_launch"] / (best / 1e3) / 1e9
    print(json.dumps(res))


def batched_case(args):
    """One batched launch over N scenes (the config-4 pattern, small)."""
    import torch

    import renderbox2_b200 as rb
    jobs, keep, alg = [], [], 0.0
    per = max(1000, args.tris // args.batched)
    rays_per = args.rays // args.batched
    for k in range(args.batched):
        sc = rb.heightfield_for_triangles(seed=300 + k, n_tris=per)
        bvh = rb.BVH(sc)
        tr = rb.CudaTracer(bvh)
        rays, _ = rb.surface_rays(sc, seed=400 + k, n=rays_per)
        d = torch.from_numpy(rays).cuda()
        h = rays_per // 2
        out_h = torch.empty((h, 4), dtype=torch.int32, device="cuda")
        out_o = torch.empty((rays_per - h,), dtype=torch.uint8, device="cuda")
        jobs += [(tr, d[:h], rb.MODE_CLOSEST, out_h, None), (tr, d[h:], rb.MODE_OCCLUSION, out_o, None)]
        keep.append((sc, bvh, tr, d, out_h, out_o, rays))
        if not args.no_oracle:
            import oracle
            nodes, woop, tri = bvh.buffers_view()
            idx = np.linspace(0, rays_per - 1, 4096).astype(np.int64)
            for mode, sl in (("ch", idx[idx < h]), ("ah", idx[idx >= h])):
                _, cnt = oracle.trace(nodes, woop, tri, rays[sl], any_hit=(mode == "ah"), counts=True)
                bpr = 32 + 64 * cnt["nodes"].astype(np.float64) + 48 * cnt["tris"] + 16 * cnt["leafterms"] + \
                    (16 if mode == "ch" else 1)
                alg += bpr.mean() * (h if mode == "ch" else rays_per - h)
    batch = rb.TraceBatch(jobs)
    batch.set_config(block_threads=args.block, regs=args.regs, node_order=args.order, fetch_threshold=28)
    ms = []
    for _ in range(args.launches):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        batch.launch()
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    assert batch.status() == 0
    res = {"scenes": args.batched, "tris_per_scene": per, "rays": rays_per * args.batched, "launch_ms": ms,
           "config": batch.config()}
    if alg:
        best = min(ms[1:] if len(ms) > 1 else ms)
        res.update(alg_bytes_per_launch=alg, achieved_gbs_best=alg / (best / 1e3) / 1e9)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
