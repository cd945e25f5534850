"""GPU tests of the serving runtime (config 5 pattern): jobs admitted while
others run overlap on the device, and every job's result is identical alone
and in the mix (bit for bit: traversal and counter-keyed sampling do not
depend on scheduling)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pool(rb, cuda):
    from renderbox2_b200.serve import build_pool
    return build_pool([5_000, 20_000, 60_000], seed=9)


def _mixed_jobs(pool):
    from renderbox2_b200.serve import JobList
    rng = np.random.Generator(np.random.PCG64(3))
    jl = JobList()
    import renderbox2_b200 as rb
    for k in range(6):
        b = k % 3
        n = int(rng.integers(10_000, 200_000))
        rays, _ = rb.surface_rays(pool.scenes[b], seed=100 + k, n=n)
        rays[::2, 4:7] *= -1.0
        jl.add_rays(b, rays, mode=0 if k % 2 == 0 else 2)
    for k in range(6):
        b = (k + 1) % 3
        tile = int(rng.integers(32, 97))
        jl.add_tile(b, tile, spp=int(rng.choice([2, 4, 8])), seed=200 + k, eye=(-0.5, 0.9, -0.3),
                    lookat=(-0.5, 0.0, 0.5))
    return jl


def _outputs_equal(a, b):
    import torch
    return all(torch.equal(x, y) for x, y in zip(a.outputs, b.outputs))


def test_results_identical_alone_and_in_the_mix(pool, cuda):
    from renderbox2_b200.serve import Server
    jobs = _mixed_jobs(pool)
    srv = Server(pool, slots=4, hbm_budget=8 << 30, max_tile=128, max_rays=256 * 1024)
    mix = jobs.subset(range(len(jobs.jobs)))
    res, st = srv.run(mix)
    assert all(r.status == 0 for r in res)
    assert st["max_concurrent"] > 1, st  # work of several jobs was in flight together
    for i in range(len(jobs.jobs)):
        alone = jobs.subset([i])
        r1, _ = srv.run(alone)
        assert r1[0].status == 0
        assert cuda.equal(alone.outputs[0], mix.outputs[i]), f"job {i} differs alone vs in the mix"
    fifo = Server(pool, fifo=True, max_tile=128, max_rays=256 * 1024)
    seq = jobs.subset(range(len(jobs.jobs)))
    rf, sf = fifo.run(seq)
    assert sf["max_concurrent"] == 1
    assert _outputs_equal(seq, mix)
    # tile images carry light (the pool scenes have an emissive panel)
    assert float(mix.outputs[-1].mean()) > 0.0


def test_ray_jobs_equal_direct_traces(pool, cuda):
    from renderbox2_b200.serve import JobList, Server
    import renderbox2_b200 as rb
    rays, _ = rb.surface_rays(pool.scenes[2], seed=55, n=50_000)
    rays[::3, 4:7] *= -1.0
    jl = JobList()
    jl.add_rays(2, rays, mode=0)
    jl.add_rays(2, rays, mode=2)
    srv = Server(pool, slots=2, max_tile=64, max_rays=64 * 1024)
    res, _ = srv.run(jl)
    d = cuda.from_numpy(rays).cuda()
    direct = pool.tracers[2].trace(d).cpu()
    occ = pool.tracers[2].trace_occlusion(d).cpu()
    assert cuda.equal(jl.outputs[0], direct)
    assert cuda.equal(jl.outputs[1], occ)


def test_admission_by_hbm_footprint(pool, cuda):
    from renderbox2_b200.serve import Server
    jobs = _mixed_jobs(pool)
    fps = [jobs.footprint(i) for i in range(len(jobs.jobs))]
    budget = max(fps) + min(fps) // 2
    srv = Server(pool, slots=8, hbm_budget=budget, max_tile=128, max_rays=256 * 1024)
    res, st = srv.run(jobs.subset(range(len(jobs.jobs))))
    assert all(r.status == 0 for r in res)
    assert st["peak_admitted_bytes"] <= budget
    # Poisson arrivals: latency is measured from arrival, never negative.
    from renderbox2_b200.serve import poisson_arrivals
    arr = poisson_arrivals(len(jobs.jobs), rate=200.0)
    res2, st2 = srv.run(jobs.with_arrivals(arr))
    assert all(r.latency_s > 0 and r.admit_s >= a - 1e-6 for r, a in zip(res2, arr))
    assert st2["p99_s"] >= st2["p50_s"] > 0


def test_shared_buffer_jobs_equal_direct_traces(pool, cuda):
    """config5_jobs over serve.SharedBuffers (the host buffers of the long
    serving runs): ray jobs read slices of one pinned ray set per BVH and every
    job writes into the circular output arena.  In a run too short to wrap the
    arena, each ray job's output equals a direct trace of its slice, and the
    continuous and the one-at-a-time servers write identical outputs."""
    from renderbox2_b200.serve import Server, SharedBuffers, _out_bytes, config5_jobs
    torch = cuda
    sh = SharedBuffers(pool, rays_per_bvh=256 * 1024, arena_bytes=1 << 30, seed=23)
    n = 24
    jobs = config5_jobs(pool, n, seed=11, tile_min=32, tile_max=96, spp_choices=(1, 2), rays_min=16 * 1024,
                        rays_max=256 * 1024, shared=sh)
    a, b = jobs.subset(range(n)), jobs.subset(range(n))
    assert 3 * sum(_out_bytes(j) + 256 for j in jobs.jobs) < sh.arena.numel()   # no wrap in this test
    base = sh.arena.data_ptr()

    def out(jl, i):
        j = jl.jobs[i]
        o = j.h_out - base
        return sh.arena[o:o + _out_bytes(j)].clone()

    ra, _ = Server(pool, slots=4, max_tile=128, max_rays=256 * 1024).run(a)
    rf, sf = Server(pool, fifo=True, max_tile=128, max_rays=256 * 1024).run(b)
    assert all(r.status == 0 for r in ra) and all(r.status == 0 for r in rf)
    assert sf["max_concurrent"] == 1
    n_ray = 0
    for i, j in enumerate(a.jobs):
        assert torch.equal(out(a, i), out(b, i)), f"job {i} differs between the servers"
        if j.kind == 0:
            n_ray += 1
            off = (j.h_rays - sh.rays[j.bvh].data_ptr()) // 32
            d = sh.rays[j.bvh][off:off + j.n_rays].cuda()
            if j.mode == 0:
                assert torch.equal(out(a, i).view(torch.int32).view(-1, 4), pool.tracers[j.bvh].trace(d).cpu())
            else:
                assert torch.equal(out(a, i), pool.tracers[j.bvh].trace_occlusion(d).cpu())
    assert 0 < n_ray < n


def test_job_deadline_times_out_one_job_and_the_loop_goes_on(pool, cuda, rb):
    """A served job whose stream is held up past its deadline (a host function
    that sleeps on the slot's stream, injected on the host) gets RB2_ETIMEOUT;
    the other jobs, admitted on the other slots meanwhile, complete with the
    same outputs as direct traces, and the run returns only after the stalled
    slot has drained."""
    import ctypes as C

    from renderbox2_b200.serve import JobList, Server
    L = rb.lib()
    L.rb2_debug_stall_next_job.argtypes = [C.c_uint32]
    jl = JobList()
    keep = []
    for k in range(10):
        rays, _ = rb.surface_rays(pool.scenes[k % 3], seed=700 + k, n=20_000)
        rays[::2, 4:7] *= -1.0
        jl.add_rays(k % 3, rays, mode=0, arrival=0.0 if k == 0 else 0.02 + 0.01 * k)
        keep.append(rays)
    srv = Server(pool, slots=3, max_tile=64, max_rays=64 * 1024, job_timeout_ms=300)
    assert L.rb2_debug_stall_next_job(1500) == 0
    res, st = srv.run(jl, raise_on_error=False)
    assert res[0].status == 6, "the stalled job must report RB2_ETIMEOUT"
    assert 0.25 < res[0].latency_s < 1.2, res[0].latency_s
    assert st["wall_s"] >= 1.4, "the run must wait for the stalled slot to drain"
    for k in range(1, 10):
        assert res[k].status == 0, (k, res[k].status)
        direct = pool.tracers[k % 3].trace(cuda.from_numpy(keep[k]).cuda()).cpu()
        assert cuda.equal(jl.outputs[k], direct), f"job {k}"
    # the server is usable afterwards, with no stall
    res2, _ = srv.run(jl.subset(range(3)))
    assert all(r.status == 0 for r in res2)


def test_server_rejects_more_slots_than_queue_heads(pool, cuda, rb):
    from renderbox2_b200._native import Rb2Error
    from renderbox2_b200.serve import Server
    with pytest.raises(Rb2Error) as e:
        Server(pool, slots=257, max_tile=64, max_rays=64 * 1024)
    assert e.value.code == 1 and "256" in str(e.value)
