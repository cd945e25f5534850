"""GPU tests of the batched job-table launch (config 4 pattern): many scenes
and uneven ray batches in one persistent launch must give exactly the
results of per-scene launches, for every launch configuration the autotuner
can pick, including graph replay and the breadth-first node order."""
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
    dict(regs=40, block_threads=64, chunk=2),
])
def test_batch_configs_give_identical_results(rb, cuda, cfg):
    scenes, tracers, jobs, outs, plain = _setup(rb, cuda)
    batch = rb.TraceBatch(jobs)
    batch.set_config(**cfg)
    for o in outs:
        o.fill_(7)
    batch.launch()
    _check(outs, plain, cuda)
    batch.set_config(node_order=0)


def test_graph_replay_and_autotune(rb, cuda):
    scenes, tracers, jobs, outs, plain = _setup(rb, cuda)
    batch = rb.TraceBatch(jobs)
    best, ms = batch.autotune(reps=2)
    assert ms > 0 and best["block_threads"] in (64, 128, 256)
    s = cuda.cuda.Stream()
    batch.capture(s)
    for _ in range(2):
        for o in outs:
            o.fill_(7)
        cuda.cuda.synchronize()
        batch.launch(s)
        s.synchronize()
        _check(outs, plain, cuda)
    batch.set_config(node_order=0)


def test_bfs_node_order_on_single_tracer(rb, cuda):
    sc = rb.heightfield_for_triangles(seed=5, n_tris=50_000)
    tr = rb.CudaTracer(rb.BVH(sc))
    r, _ = rb.surface_rays(sc, seed=6, n=100_000)
    d = cuda.from_numpy(r).cuda()
    a = tr.trace(d).clone()
    rb.lib().rb2_tracer_set_node_order(tr.handle, 1)
    b = tr.trace(d)
    assert cuda.equal(a, b)
