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
    args = ap.parse_args()

    import torch

    import renderbox2_b200 as rb
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


if __name__ == "__main__":
    main()
