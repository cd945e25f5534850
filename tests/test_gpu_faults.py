"""Device allocation failures, injected on the host (rb2_debug_fail_alloc
makes the k-th device allocation fail before cudaMalloc is called; no GPU
fault is involved).  For each create / first-use path the test fails every
allocation in turn: the entry point must return RB2_ENOMEM, free what it had
allocated (the library's live-allocation count returns to its value before),
and leave the process able to run the same path afterwards with correct
results."""
import ctypes as C
import gc

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _hooks(rb):
    L = rb.lib()
    L.rb2_debug_fail_alloc.argtypes = [C.c_uint64]
    L.rb2_debug_alloc_count.argtypes = [C.POINTER(C.c_uint64), C.POINTER(C.c_int64)]
    return L


def _live(L):
    total, live = C.c_uint64(), C.c_int64()
    assert L.rb2_debug_alloc_count(C.byref(total), C.byref(live)) == 0
    return live.value


def _sweep(rb, make, limit=300):
    """Fails allocation k = 1, 2, ... of make() until it succeeds; returns
    (number of failure points, the successful result)."""
    L = _hooks(rb)
    gc.collect()
    live0 = _live(L)
    for k in range(1, limit):
        L.rb2_debug_fail_alloc(k)
        err = None
        try:
            obj = make()
        except rb.Rb2Error as e:
            err = (e.code, str(e))
        L.rb2_debug_fail_alloc(0)
        if err is None:
            return k - 1, obj, live0
        gc.collect()
        assert err[0] == 2, f"allocation {k}: {err[1]}"
        assert _live(L) == live0, f"allocation {k} failed and {_live(L) - live0} allocations leaked ({err[1]})"
    pytest.fail("the path never succeeded")


def test_tracer_create_and_layouts(rb, orc, cuda):
    sc = rb.heightfield_scene(seed=3, grid_n=48, n_boxes=6)
    bvh = rb.BVH(sc)

    def make():
        tr = rb.CudaTracer(bvh)
        tr.set_node_order(rb.NODE_ORDER_CW8)
        tr.set_node_order(rb.NODE_ORDER_WIDE4)
        tr.set_node_order(rb.NODE_ORDER_DFS)
        return tr

    points, tr, live0 = _sweep(rb, make)
    assert points >= 4
    rays, _ = rb.surface_rays(sc, seed=4, n=20_000)
    rays[::2, 4:7] *= -1.0
    got = tr.trace(cuda.from_numpy(rays).cuda()).cpu().numpy()
    want = orc.trace(*bvh.buffers_view(), rays)
    assert np.array_equal(got[:, 0], want["prim"])
    assert tr.status() == 0
    del tr
    gc.collect()
    assert _live(_hooks(rb)) == live0


def test_batch_and_host_pipeline(rb, orc, cuda):
    sc = rb.heightfield_scene(seed=5, grid_n=32, n_boxes=4)
    bvh = rb.BVH(sc)
    tr = rb.CudaTracer(bvh)
    rays, _ = rb.surface_rays(sc, seed=6, n=30_000)
    d = cuda.from_numpy(rays).cuda()
    out_h = cuda.zeros((30_000, 4), dtype=cuda.int32, device="cuda")
    out_o = cuda.zeros((30_000,), dtype=cuda.uint8, device="cuda")
    h_rays = cuda.from_numpy(rays).pin_memory()
    h_out = cuda.zeros((30_000, 4), dtype=cuda.int32).pin_memory()

    def make():
        b = rb.TraceBatch([(tr, d, rb.MODE_CLOSEST, out_h, None), (tr, d, rb.MODE_OCCLUSION, out_o, None)])
        b.launch()
        p = rb.HostPipeline(chunk_rays=8192, depth=3)
        p.trace_jobs([(tr, h_rays, rb.MODE_CLOSEST, h_out, None)])
        return b, p

    points, (b, p), _ = _sweep(rb, make)
    assert points >= 2
    cuda.cuda.synchronize()
    want = orc.trace(*bvh.buffers_view(), rays)
    assert np.array_equal(out_h.cpu().numpy()[:, 0], want["prim"])
    assert np.array_equal(h_out.numpy()[:, 0], want["prim"])
    assert np.array_equal(out_o.cpu().numpy().astype(bool), want["prim"] >= 0)
    assert b.status() == 0


def test_integrator_renders(rb, cuda):
    from renderbox2_b200.render import (BidirectionalPathIntegratorLvcParams, DeviceScene, Integrator,
                                        PathIntegratorParams)
    room = rb.RoomScene(seed=1, n_boxes=2, n_spheres=4, sphere_subdiv=1, n_lights=1)
    tracer = rb.CudaTracer(rb.BVH(room))
    cam = rb.PerspectiveCamera((-0.5, 0.5, 0.05), (-0.5, 0.45, 1.0), (0, 1, 0), (24, 24), 60.0)
    pt = PathIntegratorParams(spp=2, max_depth=4, seed=3)
    bd = BidirectionalPathIntegratorLvcParams(spp=2, max_path_length=4, seed=3)

    def make():
        ds = DeviceScene(room)
        it = Integrator(tracer, ds)
        a = it.render_pt(cam, pt)
        b = it.render_bdpt(cam, bd)
        return ds, it, a, b

    points, (ds, it, a, b), _ = _sweep(rb, make)
    assert points >= 5
    # the same frames again, without injection: identical images
    it2 = Integrator(tracer, DeviceScene(room))
    assert cuda.equal(it2.render_pt(cam, pt), a)
    assert cuda.equal(it2.render_bdpt(cam, bd), b)


def test_server_create(rb, cuda):
    from renderbox2_b200.serve import Server, build_pool
    pool = build_pool([2_000, 5_000], seed=21)

    def make():
        return Server(pool, slots=3, max_tile=64, max_rays=32 * 1024)

    points, srv, _ = _sweep(rb, make)
    assert points >= 6
    from renderbox2_b200.serve import JobList
    jl = JobList()
    rays, _ = rb.surface_rays(pool.scenes[1], seed=9, n=10_000)
    jl.add_rays(1, rays, mode=0)
    res, _ = srv.run(jl)
    assert res[0].status == 0
    direct = pool.tracers[1].trace(cuda.from_numpy(rays).cuda()).cpu()
    assert cuda.equal(jl.outputs[0], direct)
