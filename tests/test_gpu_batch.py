"""GPU tests of the batched job-table launch (config 4 pattern): many scenes
and uneven ray batches in one persistent launch must give exactly the
results of per-scene launches, for every launch configuration the autotuner
can pick, including graph replay and the breadth-first node order.  With the
4-wide and compressed 8-wide node layouts the traversal order differs, so
closest hits must be equal except at confirmed ties, any-hit jobs must agree
on occlusion, and occlusion jobs must be byte-identical."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(rb, torch, sizes=(300, 2_000, 20_000, 120_000, 5, 60_000), rays=(70_000, 3, 150_000, 0, 1000, 90_000)):
    scenes, tracers, jobs, outs, plain = [], [], [], [], []
    modes = [rb.MODE_CLOSEST, rb.MODE_OCCLUSION, rb.MODE_ANY, rb.MODE_CLOSEST, rb.MODE_OCCLUSION, rb.MODE_CLOSEST]
    for k, (tris, n) in enumerate(zip(sizes, rays)):
        sc = rb.heightfield_for_triangles(seed=900 + k, n_tris=max(tris, 20), n_boxes=2)
        bvh = rb.BVH(sc)
        tr = rb.CudaTracer(bvh)
        r, _ = rb.surface_rays(sc, seed=950 + k, n=max(n, 1))
        r = r[:n].copy()
        r[::3, 4:7] *= -1.0  # a third of the rays point back into the surface
        d = torch.from_numpy(r).cuda()
        mode = modes[k]
        if mode == rb.MODE_OCCLUSION:
            out = torch.full((n,), 7, dtype=torch.uint8, device="cuda")
            ref = tr.trace_occlusion(d) if n else out.clone()
        else:
            out = torch.full((n, 4), 7, dtype=torch.int32, device="cuda")
            ref = tr.trace(d, any_hit=(mode == rb.MODE_ANY)) if n else out.clone()
        scenes.append((sc, bvh, r))
        tracers.append(tr)
        jobs.append((tr, d, mode, out, None))
        outs.append(out)
        plain.append(ref)
    torch.cuda.synchronize()
    return scenes, tracers, jobs, outs, plain


def _check(outs, plain, torch):
    torch.cuda.synchronize()
    for o, p in zip(outs, plain):
        assert torch.equal(o, p)


MODES = None


def _check_any_layout(rb, orc, scenes, jobs, outs, plain, torch):
    """Layout-independent equality (see the module docstring)."""
    from parity import compare_closest
    torch.cuda.synchronize()
    for (sc, bvh, r), (tr, d, mode, o, _), p in zip(scenes, jobs, plain):
        got, ref = o.cpu().numpy(), p.cpu().numpy()
        if mode == rb.MODE_OCCLUSION or r.shape[0] == 0:
            assert np.array_equal(got, ref)
        elif mode == rb.MODE_ANY:
            assert np.array_equal(got[:, 0] >= 0, ref[:, 0] >= 0)
        else:
            nodes, woop, tri = bvh.buffers_view()
            f = ref.view(np.float32)
            want = {"prim": ref[:, 0], "t": f[:, 1], "u": f[:, 2], "v": f[:, 3]}
            ties, bad, first = compare_closest(orc, got, want, woop, tri, r)
            assert bad == 0, f"ray {first}"


def test_batch_equals_plain_launches(rb, orc, cuda):
    scenes, tracers, jobs, outs, plain = _setup(rb, cuda)
    batch = rb.TraceBatch(jobs)
    batch.launch()
    _check(outs, plain, cuda)
    assert batch.status() == 0
    # and the plain launches equal the oracle (closest-hit job 0)
    sc, bvh, r = scenes[0]
    want = orc.trace(*bvh.buffers_view(), r)
    got = outs[0].cpu().numpy()
    assert np.array_equal(got[:, 0], want["prim"])
    assert np.array_equal(got[:, 1].view(np.float32).view(np.uint32), want["t"].view(np.uint32))


@pytest.mark.parametrize("cfg", [
    dict(block_threads=64), dict(block_threads=256), dict(chunk=4), dict(chunk=8, fetch_threshold=8),
    dict(node_order=1), dict(ctas_per_sm=2, fetch_threshold=32), dict(regs=48), dict(regs=40, block_threads=256),
    dict(regs=40, block_threads=64, chunk=2), dict(node_order=2), dict(node_order=2, regs=48, block_threads=256),
    dict(node_order=2, regs=40, chunk=4), dict(node_order=3), dict(node_order=3, regs=48, block_threads=256),
    dict(node_order=3, regs=40, chunk=4, fetch_threshold=8),
    dict(reorder=3), dict(reorder=4, chunk=4), dict(reorder=5, node_order=1, regs=48, block_threads=256),
    dict(reorder=4, node_order=2), dict(reorder=4, node_order=3, regs=48, block_threads=256, fetch_threshold=16),
    dict(reorder=5, node_order=3, regs=40, chunk=2), dict(reorder=6), dict(reorder=6, node_order=3, regs=48),
    dict(node_threshold=1), dict(node_order=1, node_threshold=8, reorder=4), dict(node_order=2, node_threshold=16),
    dict(node_order=3, node_threshold=1), dict(node_order=3, node_threshold=32, block_threads=64),
    dict(node_order=3, node_threshold=4, reorder=4, fetch_threshold=28),
])
def test_batch_configs_give_identical_results(rb, orc, cuda, cfg):
    scenes, tracers, jobs, outs, plain = _setup(rb, cuda)
    batch = rb.TraceBatch(jobs)
    batch.set_config(**cfg)
    for o in outs:
        o.fill_(7)
    batch.launch()
    if cfg.get("node_order") in (2, 3):
        _check_any_layout(rb, orc, scenes, jobs, outs, plain, cuda)
    else:
        _check(outs, plain, cuda)
    assert batch.status() == 0
    batch.set_config(node_order=0)


def test_graph_replay_and_autotune(rb, orc, cuda):
    scenes, tracers, jobs, outs, plain = _setup(rb, cuda)
    batch = rb.TraceBatch(jobs)
    best, ms = batch.autotune(reps=2)
    assert ms > 0 and best["block_threads"] in (64, 128, 256) and best["node_order"] in (0, 1, 2, 3)
    s = cuda.cuda.Stream()
    batch.capture(s)
    for _ in range(2):
        for o in outs:
            o.fill_(7)
        cuda.cuda.synchronize()
        batch.launch(s)
        s.synchronize()
        _check_any_layout(rb, orc, scenes, jobs, outs, plain, cuda)
    batch.set_config(node_order=0)


def test_wide_layout_single_tracer_and_layout_guard(rb, orc, cuda):
    """A tracer switched to the 4-wide layout traces like the binary one
    (closest hits equal but for confirmed ties, occlusion identical); a batch
    whose tracer was switched by someone else refuses to launch until its
    configuration is set again."""
    from parity import compare_closest
    sc = rb.heightfield_for_triangles(seed=15, n_tris=300_000, n_boxes=40)
    bvh = rb.BVH(sc)
    tr = rb.CudaTracer(bvh)
    r, _ = rb.surface_rays(sc, seed=16, n=200_000)
    d = cuda.from_numpy(r).cuda()
    a = tr.trace(d).cpu().numpy()
    occ_a = tr.trace_occlusion(d).cpu().numpy()
    assert rb.lib().rb2_tracer_set_node_order(tr.handle, 2) == 0
    b = tr.trace(d).cpu().numpy()
    occ_b = tr.trace_occlusion(d).cpu().numpy()
    assert np.array_equal(occ_a, occ_b)
    nodes, woop, tri = bvh.buffers_view()
    f = a.view(np.float32)
    ties, bad, first = compare_closest(orc, b, {"prim": a[:, 0], "t": f[:, 1], "u": f[:, 2], "v": f[:, 3]}, woop, tri, r)
    assert bad == 0, f"ray {first}"
    want = orc.trace(nodes, woop, tri, r)
    ties, bad, first = compare_closest(orc, b, {k: want[k] for k in ("prim", "t", "u", "v")}, woop, tri, r)
    assert bad == 0, f"ray {first} vs oracle"
    # integrator-facing device view stays binary
    assert tr.get_bvh()["n_nodes_u4"] == nodes.shape[0]
    out = cuda.empty((1000, 4), dtype=cuda.int32, device="cuda")
    batch = rb.TraceBatch([(tr, d[:1000], rb.MODE_CLOSEST, out, None)])
    batch.launch()
    assert rb.lib().rb2_tracer_set_node_order(tr.handle, 0) == 0
    with pytest.raises(rb.Rb2Error, match="layout"):
        batch.launch()
    batch.set_config(node_order=0)
    batch.launch()
    cuda.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), a[:1000])


def test_bfs_node_order_on_single_tracer(rb, cuda):
    sc = rb.heightfield_for_triangles(seed=5, n_tris=50_000)
    tr = rb.CudaTracer(rb.BVH(sc))
    r, _ = rb.surface_rays(sc, seed=6, n=100_000)
    d = cuda.from_numpy(r).cuda()
    a = tr.trace(d).clone()
    rb.lib().rb2_tracer_set_node_order(tr.handle, 1)
    b = tr.trace(d)
    assert cuda.equal(a, b)


@pytest.mark.parametrize("seed,n_tris,n_boxes,n_rays", [(15, 300_000, 40, 200_000), (21, 4_000, 64, 100_000)])
def test_cw8_layout_single_tracer(rb, orc, cuda, seed, n_tris, n_boxes, n_rays):
    """A tracer switched to the compressed 8-wide layout: closest hits equal
    the oracle's but for confirmed ties, occlusion is byte-identical, the
    status word stays clean, and switching back restores the binary results."""
    from parity import compare_closest
    sc = rb.heightfield_for_triangles(seed=seed, n_tris=n_tris, n_boxes=n_boxes)
    bvh = rb.BVH(sc)
    tr = rb.CudaTracer(bvh)
    r, _ = rb.surface_rays(sc, seed=seed + 1, n=n_rays)
    r[::4, 4:7] *= -1.0
    d = cuda.from_numpy(r).cuda()
    a = tr.trace(d).cpu().numpy()
    occ_a = tr.trace_occlusion(d).cpu().numpy()
    assert rb.lib().rb2_tracer_set_node_order(tr.handle, rb.NODE_ORDER_CW8) == 0
    b = tr.trace(d).cpu().numpy()
    occ_b = tr.trace_occlusion(d).cpu().numpy()
    anyh = tr.trace(d, any_hit=True).cpu().numpy()
    assert tr.status() == 0
    assert np.array_equal(occ_a, occ_b)
    assert np.array_equal(anyh[:, 0] >= 0, a[:, 0] >= 0)
    nodes, woop, tri = bvh.buffers_view()
    want = orc.trace(nodes, woop, tri, r)
    ties, bad, first = compare_closest(orc, b, {k: want[k] for k in ("prim", "t", "u", "v")}, woop, tri, r)
    print("cw8 ties", ties)
    assert bad == 0, f"ray {first} vs oracle"
    assert rb.lib().rb2_tracer_set_node_order(tr.handle, rb.NODE_ORDER_DFS) == 0
    assert np.array_equal(tr.trace(d).cpu().numpy(), a)


def test_cw8_layout_with_ref_list_nodes(rb, orc, cuda):
    """Leaves of hundreds of coincident triangles go into the compressed
    layout's ref-list nodes: closest hits still equal the oracle's (ties
    confirmed), occlusion is identical."""
    from parity import compare_closest
    from test_cw8_layout import _degenerate_scene, _rays_at_cluster
    bvh = rb.BVH(_degenerate_scene(rb))
    tr = rb.CudaTracer(bvh)
    r = _rays_at_cluster(50_000, 7)
    d = cuda.from_numpy(r).cuda()
    occ_a = tr.trace_occlusion(d).cpu().numpy()
    tr.set_node_order(rb.NODE_ORDER_CW8)
    b = tr.trace(d).cpu().numpy()
    assert np.array_equal(tr.trace_occlusion(d).cpu().numpy(), occ_a)
    assert tr.status() == 0
    nodes, woop, tri = bvh.buffers_view()
    want = orc.trace(nodes, woop, tri, r)
    ties, bad, first = compare_closest(orc, b, {k: want[k] for k in ("prim", "t", "u", "v")}, woop, tri, r)
    print("cw8 ref-list ties", ties)
    assert bad == 0, f"ray {first}"


def test_cw8_layout_on_rooms(rb, orc, cuda):
    """Rooms (flat wall and box leaves, spheres) through the compressed layout:
    closest hits equal the oracle's but for confirmed ties, occlusion is
    byte-identical to the binary layout's."""
    from parity import compare_closest
    for seed in (4, 5):
        sc = rb.RoomScene(seed=seed, n_boxes=20, n_spheres=200, sphere_subdiv=2, n_lights=2)
        bvh = rb.BVH(sc)
        tr = rb.CudaTracer(bvh)
        r, _ = rb.surface_rays(sc, seed=seed + 10, n=200_000)
        d = cuda.from_numpy(r).cuda()
        occ_a = tr.trace_occlusion(d).cpu().numpy()
        tr.set_node_order(rb.NODE_ORDER_CW8)
        b = tr.trace(d).cpu().numpy()
        assert np.array_equal(tr.trace_occlusion(d).cpu().numpy(), occ_a)
        assert tr.status() == 0
        nodes, woop, tri = bvh.buffers_view()
        want = orc.trace(nodes, woop, tri, r)
        ties, bad, first = compare_closest(orc, b, {k: want[k] for k in ("prim", "t", "u", "v")}, woop, tri, r)
        assert bad == 0, f"seed {seed}, ray {first}"


def test_ray_reordering_keeps_every_ray(rb, orc, cuda):
    """Ray reordering visits each job's rays in (octant, Morton code of the
    origin) order: with stencil masks, origins far outside the scene box,
    empty and one-ray jobs and a job spanning two scenes' worth of rays, every
    record still lands at its own ray's index and equals the plain launch's,
    for 3 to 6 bits per axis (one- and two-pass sorts) and after graph
    capture; widths outside 3..6 are refused."""
    scenes, tracers, jobs, outs, plain = _setup(rb, cuda)
    # job 0 gets a stencil and a block of rays whose origins sit far outside the box
    sc, bvh, r = scenes[0]
    far = r.copy()
    far[:5000, 0:3] += np.float32(50.0)
    far[5000:6000, 0:3] -= np.float32(1e4)
    d_far = cuda.from_numpy(far).cuda()
    mask = cuda.from_numpy((np.arange(far.shape[0]) % 5 != 2).astype(np.uint8)).cuda()
    out_m = cuda.full((far.shape[0], 4), 7, dtype=cuda.int32, device="cuda")
    ref_m = tracers[0].trace(d_far, stencil=mask).clone()
    jobs = jobs + [(tracers[0], d_far, rb.MODE_CLOSEST, out_m, mask)]
    outs = outs + [out_m]
    plain = plain + [ref_m]
    batch = rb.TraceBatch(jobs)
    for bits in (3, 4, 5, 6):
        batch.set_config(reorder=bits)
        for o in outs:
            o.fill_(7)
        batch.launch()
        _check(outs, plain, cuda)
        assert batch.status() == 0
    s = cuda.cuda.Stream()
    batch.capture(s)
    for _ in range(2):
        for o in outs:
            o.fill_(7)
        cuda.cuda.synchronize()
        batch.launch(s)
        s.synchronize()
        _check(outs, plain, cuda)
    for bad in (1, 2, 7):
        with pytest.raises(rb.Rb2Error, match="reorder"):
            batch.set_config(reorder=bad)
    # the masked job equals the oracle on its active rays
    nodes, woop, tri = bvh.buffers_view()
    act = mask.cpu().numpy() != 0
    want = orc.trace(nodes, woop, tri, far[act])
    got = out_m.cpu().numpy()[act]
    assert np.array_equal(got[:, 0], want["prim"])
    assert np.array_equal(got[:, 1].view(np.uint32), want["t"].view(np.uint32))


def test_ray_reordering_refused_for_many_tiny_jobs(rb, cuda):
    """A batch of 3,000 jobs of 5 rays each would need far more sort counters
    than it has rays: every reordering width is refused with a clear error,
    the autotuner leaves reordering off, and the launch still equals the
    plain trace."""
    sc = rb.heightfield_for_triangles(seed=77, n_tris=2_000)
    tr = rb.CudaTracer(rb.BVH(sc))
    r, _ = rb.surface_rays(sc, seed=78, n=15_000)
    d = cuda.from_numpy(r).cuda()
    out = cuda.full((r.shape[0], 4), 7, dtype=cuda.int32, device="cuda")
    jobs = [(tr, d[5 * k: 5 * k + 5], rb.MODE_CLOSEST, out[5 * k: 5 * k + 5], None) for k in range(3000)]
    batch = rb.TraceBatch(jobs)
    for bits in (3, 4, 5, 6):
        with pytest.raises(rb.Rb2Error, match="reordering"):
            batch.set_config(reorder=bits)
    best, ms = batch.autotune(reps=1)
    assert best["reorder"] == 0 and ms > 0
    out.fill_(7)
    batch.launch()
    cuda.cuda.synchronize()
    ref = tr.trace(d)
    if best["node_order"] in (2, 3):
        assert cuda.equal(out[:, 0] >= 0, ref[:, 0] >= 0)
    else:
        assert cuda.equal(out, ref)
    assert batch.status() == 0
