"""GPU parity of the traversal kernel and camera rays (B200), through the C ABI.

Bar: closest-hit prim, t, u, v bit-identical to the CPU oracle on the same
buffers and rays; mismatches are allowed only at ties (two triangles that
accept the ray at exactly the same t) and are counted.  Any-hit occlusion
decisions must match exactly."""
import numpy as np
import pytest

from parity import compare_any, compare_closest, golden

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _oracle_dict(h):
    return {"prim": h["prim"], "t": h["t"], "u": h["u"], "v": h["v"]}


def test_golden_fixture_closest_and_any_hit(rb, orc, cuda):
    g = golden()
    bvh = rb.BVH.from_buffers(g["ref_nodes"], g["ref_woop"], g["ref_triidx"])
    tr = rb.CudaTracer(bvh)
    rays = _dev(cuda, g["rays"])
    got = tr.trace(rays).cpu().numpy()
    ref = {"prim": g["ch_prim"], "t": g["ch_t"], "u": g["ch_u"], "v": g["ch_v"]}
    ties, bad, first = compare_closest(orc, got, ref, g["ref_woop"], g["ref_triidx"], g["rays"])
    assert bad == 0, f"ray {first}: gpu {got[first]} vs golden prim {g['ch_prim'][first]}"
    ah = tr.trace(rays, any_hit=True).cpu().numpy()
    assert compare_any(ah, {"prim": g["ah_prim"]}) == 0
    occ = tr.trace_occlusion(rays).cpu().numpy()
    assert np.array_equal(occ.astype(bool), g["ah_prim"] >= 0)
    assert tr.status() == 0


@pytest.mark.parametrize("tree", ["reference", "rb2"])
def test_incoherent_rays_match_oracle(rb, orc, cuda, tree):
    scene = rb.heightfield_scene(seed=31, grid_n=96, n_boxes=24)
    if tree == "reference":
        if not orc.have_ref():
            pytest.skip("oracle/_ref not built")
        r = orc.ref_build(scene.vertices, scene.indices)
        bvh = rb.BVH.from_buffers(r["nodes"], r["woop"], r["triidx"])
    else:
        bvh = rb.BVH(scene)
    nodes, woop, tri = bvh.get_node_buffer(), bvh.get_tri_woop_buffer(), bvh.get_tri_index_buffer()
    rays, _ = rb.surface_rays(scene, seed=32, n=300_000)
    # Half the rays point back into the surface so most of them hit.
    rays[::2, 4:7] *= -1.0
    tr = rb.CudaTracer(bvh)
    d = _dev(cuda, rays)
    got = tr.trace(d).cpu().numpy()
    want = orc.trace(nodes, woop, tri, rays)
    ties, bad, first = compare_closest(orc, got, _oracle_dict(want), woop, tri, rays)
    assert bad == 0, f"ray {first}: gpu {got[first]} vs oracle {want[first]}"
    assert (want["prim"] >= 0).mean() > 0.4
    got_ah = tr.trace(d, any_hit=True).cpu().numpy()
    want_ah = orc.trace(nodes, woop, tri, rays, any_hit=True)
    assert compare_any(got_ah, _oracle_dict(want_ah)) == 0
    print(f"{tree}: ties {ties} of {rays.shape[0]}")


def test_rb2_tree_against_reference_tree_oracle(rb, orc, cuda):
    """GPU on rb2's own SBVH vs the oracle on the reference's SBVH."""
    if not orc.have_ref():
        pytest.skip("oracle/_ref not built")
    scene = rb.RoomScene(seed=33, n_boxes=10, n_spheres=40, sphere_subdiv=2, n_lights=1)
    r = orc.ref_build(scene.vertices, scene.indices)
    rays, _ = rb.surface_rays(scene, seed=34, n=100_000)
    want = orc.trace(r["nodes"], r["woop"], r["triidx"], rays)
    tr = rb.CudaTracer(rb.BVH(scene))
    got = tr.trace(_dev(cuda, rays)).cpu().numpy()
    ties, bad, first = compare_closest(orc, got, _oracle_dict(want), r["woop"], r["triidx"], rays)
    assert bad == 0, f"ray {first}"
    assert (want["prim"] >= 0).mean() > 0.95  # closed room: nearly every ray hits


def test_camera_rays_bit_exact_with_reference_camera(rb, cuda):
    from renderbox2_b200.configs import CONFIG1 as C1
    g = golden()
    cam = rb.PerspectiveCamera(C1["eye"], C1["lookat"], C1["up"], (C1["width"], C1["height"]), C1["fov"])
    got = cam.generate_rays_at(_dev(cuda, g["cam_xy"])).cpu().numpy()
    assert np.array_equal(got.view(np.uint32), g["cam_rays"].view(np.uint32))
    # Pixel-centre grid: ray for pixel p is the camera ray at (p % w + .5, p // w + .5).
    full = cam.generate_rays().cpu().numpy()
    pix = np.array([0, 1, 511, 512, 130_000, 262_143])
    xy = np.stack([(pix % 512) + 0.5, (pix // 512) + 0.5], 1).astype(np.float32)
    at = cam.generate_rays_at(_dev(cuda, xy)).cpu().numpy()
    assert np.array_equal(full[pix].view(np.uint32), at.view(np.uint32))


def test_mask_empty_and_host_path(rb, orc, cuda):
    g = golden()
    bvh = rb.BVH.from_buffers(g["ref_nodes"], g["ref_woop"], g["ref_triidx"])
    tr = rb.CudaTracer(bvh)
    rays = g["rays"]
    mask = (np.arange(rays.shape[0]) % 3 != 0).astype(np.uint8)
    got = tr.trace(_dev(cuda, rays), stencil=_dev(cuda, mask)).cpu().numpy()
    want = orc.trace(g["ref_nodes"], g["ref_woop"], g["ref_triidx"], rays, mask=mask)
    assert np.array_equal(got[:, 0], want["prim"])
    assert (got[mask == 0, 0] == -1).all()
    # Empty batch is a no-op.
    tr.trace(_dev(cuda, rays[:0].copy()))
    # Host-buffer path equals the device path.
    host = tr.trace_host(rays)
    dev = tr.trace(_dev(cuda, rays)).cpu().numpy()
    assert np.array_equal(host, dev)
    host_m = tr.trace_host(rays, stencil=mask)
    assert np.array_equal(host_m, got)


@pytest.mark.parametrize("chunk,depth", [(1000, 3), (1 << 20, 1), (777, 16)])
def test_pipelined_host_jobs_match_oracle(rb, orc, cuda, chunk, depth):
    """rb2_trace_host_jobs over two scenes x three modes, ragged chunking
    (chunk boundaries inside jobs, last chunk short), masks on some jobs,
    an empty job: every output equals the oracle's."""
    torch = cuda
    pipe = rb.HostPipeline(chunk_rays=chunk, depth=depth)
    jobs, want = [], []
    for k, (n_tris, n) in enumerate([(20_000, 4099), (3_000, 2500)]):
        sc = rb.heightfield_for_triangles(seed=900 + k, n_tris=n_tris)
        bvh = rb.BVH(sc)
        tr = rb.CudaTracer(bvh)
        nodes, woop, tri = bvh.buffers_view()
        rays, _ = rb.surface_rays(sc, seed=910 + k, n=n)
        mask = (np.arange(n) % 5 != 1).astype(np.uint8)
        pinned = torch.from_numpy(rays).pin_memory()
        for mode, m in ((rb.MODE_CLOSEST, None), (rb.MODE_ANY, mask), (rb.MODE_OCCLUSION, mask)):
            if mode == rb.MODE_OCCLUSION:
                out = torch.full((n,), 7, dtype=torch.uint8).pin_memory()
            else:
                out = torch.full((n, 4), 7, dtype=torch.int32).pin_memory()
            jobs.append((tr, pinned, mode, out, None if m is None else torch.from_numpy(m)))
            ref = orc.trace(nodes, woop, tri, rays, any_hit=mode != rb.MODE_CLOSEST, mask=m)
            want.append((mode, ref, nodes, woop, tri, rays, out))
    empty_out = torch.full((1, 4), 7, dtype=torch.int32)
    jobs.append((jobs[0][0], torch.empty((0, 8), dtype=torch.float32), rb.MODE_CLOSEST, empty_out, None))
    pipe.trace_jobs(jobs)
    for mode, ref, nodes, woop, tri, rays, out in want:
        got = out.numpy()
        if mode == rb.MODE_CLOSEST:
            ties, bad, first = compare_closest(orc, got, _oracle_dict(ref), woop, tri, rays)
            assert bad == 0, f"ray {first}"
        elif mode == rb.MODE_ANY:
            assert compare_any(got, ref) == 0
        else:
            assert np.array_equal(got.astype(bool), ref["prim"] >= 0)
    assert (empty_out.numpy() == 7).all()
    for j in jobs:
        assert j[0].status() == 0


def test_config1_full_size(rb, orc, cuda):
    """Config 1 at full size (131,840 triangles, 512x512 primary rays, 4M
    diffuse rays): primary rays bit-exact against the oracle; for the 4M
    set a 200k sample is compared and any-hit must equal "closest hit exists"
    on every ray."""
    from renderbox2_b200.configs import CONFIG1 as C1
    scene = rb.heightfield_scene(seed=C1["seed"], grid_n=C1["grid_n"], amplitude=C1["amplitude"],
                                 n_boxes=C1["n_boxes"], box_min=C1["box_min"], box_max=C1["box_max"])
    assert scene.num_triangles == 131_840
    bvh = rb.BVH(scene)
    tr = rb.CudaTracer(bvh)
    nodes, woop, tri = bvh.get_node_buffer(), bvh.get_tri_woop_buffer(), bvh.get_tri_index_buffer()
    cam = rb.PerspectiveCamera(C1["eye"], C1["lookat"], C1["up"], (C1["width"], C1["height"]), C1["fov"])
    prim = cam.generate_rays()
    got = tr.trace(prim).cpu().numpy()
    prim_h = prim.cpu().numpy()
    want = orc.trace(nodes, woop, tri, prim_h)
    ties, bad, first = compare_closest(orc, got, _oracle_dict(want), woop, tri, prim_h)
    assert bad == 0, f"primary ray {first}"
    assert (want["prim"] >= 0).mean() > 0.5
    rays, _ = rb.surface_rays(scene, seed=41, n=4 * 1024 * 1024)
    d = _dev(cuda, rays)
    ch = tr.trace(d).cpu().numpy()
    ah = tr.trace(d, any_hit=True).cpu().numpy()
    assert np.array_equal(ch[:, 0] >= 0, ah[:, 0] >= 0)
    sel = np.random.Generator(np.random.PCG64(5)).choice(rays.shape[0], 200_000, replace=False)
    want = orc.trace(nodes, woop, tri, rays[sel])
    ties, bad, first = compare_closest(orc, ch[sel], _oracle_dict(want), woop, tri, rays[sel])
    assert bad == 0
