"""Generates the committed golden fixtures in this directory.

Run from the repository root with the reference sources present:
    make -C oracle && python -m renderbox2_b200.build && python tests/golden/make_golden.py

Everything that defines an expected value here comes from the reference's own
code compiled in place (oracle/_ref/librb2ref.so): its SBVH builder and
Compact2 packer (accelerators/sbvh/splitbvhbuilder.cpp, cudabvh.cpp), its text
cache writer (cudabvh.cpp:176-214), its perspective camera (core/camera.cu)
and its host Moller-Trumbore test (core/primitives.cu:51-70).  Hit records
are the CPU restatement of trace_ray run on the reference-built buffers; the
fixture pins that restatement so later changes to it are caught.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

import oracle  # noqa: E402
import renderbox2_b200 as rb  # noqa: E402
from renderbox2_b200.configs import CONFIG1  # noqa: E402


def main():
    if not oracle.have_ref():
        raise SystemExit("oracle/_ref/librb2ref.so missing: run `make -C oracle ref` with the reference present")
    scene = rb.heightfield_scene(seed=11, grid_n=16, amplitude=0.2, n_boxes=4, box_min=0.02, box_max=0.1)
    ref = oracle.ref_build(scene.vertices, scene.indices, cache_path=str(HERE / "ref_cache_small.txt"))
    surf, _ = rb.surface_rays(scene, seed=12, n=2048)
    xy = np.random.Generator(np.random.PCG64(13)).uniform(0.0, 512.0, size=(1024, 2)).astype(np.float32)
    cam = oracle.ref_camera_rays(CONFIG1["eye"], CONFIG1["lookat"], CONFIG1["up"], CONFIG1["width"],
                                 CONFIG1["height"], CONFIG1["fov"], xy)
    rays = np.concatenate([surf, cam]).astype(np.float32)
    ch, cnt = oracle.trace(ref["nodes"], ref["woop"], ref["triidx"], rays, any_hit=False, counts=True, nthreads=1)
    ah = oracle.trace(ref["nodes"], ref["woop"], ref["triidx"], rays, any_hit=True, nthreads=1)
    # Reference Moller-Trumbore on the closest-hit triangle of every hit ray.
    mt_uvt = np.zeros((rays.shape[0], 3), np.float32)
    mt_hit = np.zeros((rays.shape[0],), np.uint8)
    for k in np.nonzero(ch["prim"] >= 0)[0]:
        tri = scene.indices[ch["prim"][k]]
        ok, uvt = oracle.ref_intersect_triangle(scene.vertices[tri[0]], scene.vertices[tri[1]],
                                                scene.vertices[tri[2]], rays[k])
        mt_hit[k] = ok
        mt_uvt[k] = uvt
    np.savez_compressed(
        HERE / "golden_small.npz",
        vertices=scene.vertices, indices=scene.indices,
        ref_nodes=ref["nodes"], ref_woop=ref["woop"], ref_triidx=ref["triidx"], ref_sah=np.float32(ref["sah"]),
        rays=rays, cam_xy=xy, cam_rays=cam,
        ch_prim=ch["prim"], ch_t=ch["t"], ch_u=ch["u"], ch_v=ch["v"],
        ch_nodes=cnt["nodes"], ch_tris=cnt["tris"], ch_terms=cnt["leafterms"],
        ah_prim=ah["prim"], ah_t=ah["t"],
        mt_hit=mt_hit, mt_uvt=mt_uvt,
    )
    print("wrote", HERE / "golden_small.npz", "hits:", int((ch["prim"] >= 0).sum()), "of", rays.shape[0])


if __name__ == "__main__":
    main()
