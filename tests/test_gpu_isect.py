"""GPU parity of the intersection-record trace (rb2_trace_isect) and of the
header-only device traversal (rb2_trace_per_thread), through the C ABI.

Bar: every field of the SoA intersection record bit-identical to the oracle's
restatement (oracle.isect over oracle.trace hits), which is itself pinned to
the reference's compute_normal and Ray::operator() (test_oracle.py).  The
per-thread traversal follows the oracle's single-lane order exactly, so its
hit records must equal the oracle's with no tie allowance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _room(rb):
    return rb.RoomScene(seed=41, n_boxes=12, n_spheres=30, sphere_subdiv=2, n_lights=2)


def _rays(rb, scene, n, seed):
    rays, _ = rb.surface_rays(scene, seed=seed, n=n)
    # Shorten a third of the rays so some miss (tmax below the first hit).
    rays[::3, 7] = 1e-3
    return np.ascontiguousarray(rays)


def _tris4(scene):
    ix = np.asarray(scene.indices, np.uint32).reshape(-1, 3)
    m = np.asarray(scene.material_ids, np.uint32).reshape(-1)
    return np.concatenate([ix, m[:, None]], 1)


def _bits(x):
    return np.ascontiguousarray(x).view(np.uint32)


@pytest.mark.parametrize("masked,order", [(False, 0), (True, 0), (False, 3), (True, 3)])
def test_trace_isect_closest_matches_oracle(rb, orc, cuda, masked, order):
    """order 3: the tracer on the compressed 8-wide layout, which
    rb2_trace_isect then traverses."""
    from renderbox2_b200.render import DeviceScene, trace_isect
    torch = cuda
    scene = _room(rb)
    bvh = rb.BVH(scene)
    tr = rb.CudaTracer(bvh)
    tr.set_node_order(order)
    ds = DeviceScene(scene)
    nodes, woop, tri = bvh.buffers_view()
    rays = _rays(rb, scene, 20_011, seed=42)
    mask = (np.arange(rays.shape[0]) % 7 != 3).astype(np.uint8) if masked else None
    out = trace_isect(tr, ds, torch.from_numpy(rays).cuda(), any_hit=False,
                      stencil=None if mask is None else torch.from_numpy(mask).cuda())
    torch.cuda.synchronize()
    hits = orc.trace(nodes, woop, tri, rays, mask=mask)
    want = orc.isect(np.asarray(scene.vertices, np.float32), _tris4(scene), rays, hits)
    hit = hits["prim"] >= 0
    assert 0.2 < hit.mean() < 0.9
    got = {k: v.cpu().numpy() for k, v in out.t.items()}
    assert np.array_equal(got["intersected"], hit.astype(np.uint8))
    # Rays whose record differs anywhere must be ties (two triangles accepting
    # the ray at the same t, reported in a different order); there the record
    # is the oracle's record of the GPU's triangle.
    gp = got["primitive_id"].view(np.uint32)
    tie = np.zeros(hit.shape, bool)
    slots = orc.woop_slots_of(woop, tri) if (gp[hit] != want["prim"][hit]).any() else {}
    for i in np.nonzero(hit & (gp != want["prim"]))[0]:
        assert orc.is_tie(woop, tri, slots, rays[i], int(gp[i]), int(want["prim"][i])), f"ray {i}"
        tie[i] = True
    if tie.any():
        h2 = hits.copy()
        h2["prim"][tie] = gp[tie].astype(np.int32)
        want = orc.isect(np.asarray(scene.vertices, np.float32), _tris4(scene), rays, h2)
    # Ties are rare and all confirmed above; the compressed layout visits
    # leaves in another order, so it reports the other triangle more often.
    assert tie.sum() <= (max(2, hit.sum() // 10000) if order == 0 else max(16, hit.sum() // 500))
    for k_got, k_want in (("position", "position"), ("geometric_normal", "ng"), ("shading_normal", "ns"),
                          ("incoming_direction", "wi")):
        assert np.array_equal(_bits(got[k_got][:, hit]), _bits(want[k_want][:, hit])), k_got
        assert np.isnan(got[k_got][:, ~hit]).all(), f"{k_got} written on a miss"
    assert np.array_equal(_bits(got["uv"][hit & ~tie]), _bits(want["uv"][hit & ~tie]))
    assert np.array_equal(gp[hit], want["prim"][hit])
    assert np.array_equal(got["primitive_material_id"][hit].view(np.uint32), want["material"][hit])
    assert np.array_equal(got["front"][hit], want["front"][hit])
    assert np.array_equal(_bits(got["epsilon"][hit]), _bits(want["epsilon"][hit]))
    assert (got["front"][~hit] == 0xFF).all() and (got["primitive_id"][~hit] == -1).all()
    # Where the ray is traced, the record agrees with the bulk trace's hit flag.
    plain = tr.trace(torch.from_numpy(rays).cuda()).cpu().numpy()
    live = np.ones(hit.shape, bool) if mask is None else mask == 1
    assert np.array_equal((plain[:, 0] >= 0)[live], hit[live])
    assert tr.status() == 0


def test_trace_isect_any_hit_and_field_subset(rb, orc, cuda):
    from renderbox2_b200.render import DeviceScene, IntersectionBuffer, trace_isect
    torch = cuda
    scene = _room(rb)
    bvh = rb.BVH(scene)
    tr = rb.CudaTracer(bvh)
    ds = DeviceScene(scene)
    nodes, woop, tri = bvh.buffers_view()
    rays = _rays(rb, scene, 9_000, seed=43)
    d = torch.from_numpy(rays).cuda()
    # Any hit (the reference's default): only `intersected` is written.
    out = trace_isect(tr, ds, d)
    torch.cuda.synchronize()
    ah = orc.trace(nodes, woop, tri, rays, any_hit=True)
    assert np.array_equal(out["intersected"].cpu().numpy(), (ah["prim"] >= 0).astype(np.uint8))
    assert torch.isnan(out["position"]).all() and (out["primitive_id"] == -1).all()
    # Closest hit writing only two fields.
    sub = IntersectionBuffer(rays.shape[0], d.device, fields=("primitive_id", "intersected"))
    trace_isect(tr, ds, d, any_hit=False, out=sub)
    ch = orc.trace(nodes, woop, tri, rays)
    got = sub["primitive_id"].cpu().numpy()
    hit = ch["prim"] >= 0
    assert (got[~hit] == -1).all() and (got[hit] >= 0).all()
    slots = orc.woop_slots_of(woop, tri)
    for i in np.nonzero(hit & (got != ch["prim"]))[0]:
        assert orc.is_tie(woop, tri, slots, rays[i], int(got[i]), int(ch["prim"][i])), f"ray {i}"
    # Empty batch is a no-op; a vector field with a missing plane is rejected.
    trace_isect(tr, ds, d[:0])
    bad = IntersectionBuffer(4, d.device, fields=("position",))
    b = bad.c_struct()
    b.position[2] = None
    import ctypes as C

    from renderbox2_b200._native import lib
    assert lib().rb2_trace_isect(tr.handle, ds.handle, d.data_ptr(), 4, 0, None, C.byref(b), None) != 0
    assert tr.status() == 0


@pytest.mark.parametrize("any_hit", [False, True])
def test_per_thread_device_traversal_equals_oracle(rb, orc, cuda, any_hit):
    torch = cuda
    for k, n_tris in enumerate((2_000, 200_000)):
        scene = rb.heightfield_for_triangles(seed=60 + k, n_tris=n_tris)
        bvh = rb.BVH(scene)
        tr = rb.CudaTracer(bvh)
        nodes, woop, tri = bvh.buffers_view()
        rays, _ = rb.surface_rays(scene, seed=70 + k, n=30_000)
        mask = (np.arange(rays.shape[0]) % 11 != 5).astype(np.uint8)
        got = tr.trace_per_thread(torch.from_numpy(rays).cuda(), any_hit=any_hit,
                                  stencil=torch.from_numpy(mask).cuda()).cpu().numpy()
        want = orc.trace(nodes, woop, tri, rays, any_hit=any_hit, mask=mask)
        assert np.array_equal(got[:, 0], want["prim"])
        f = got.view(np.float32)
        for j, name in ((1, "t"), (2, "u"), (3, "v")):
            assert np.array_equal(_bits(f[:, j]), _bits(want[name])), name
    info = tr.get_bvh()
    assert info["n_nodes_u4"] == nodes.shape[0] and info["nodes"] % 16 == 0


def test_cpp_headers_from_user_cuda_code(rb, cuda, tmp_path):
    """A user program compiled with nvcc against include/: rb2.hpp's
    CudaTracer::trace with a reference-layout IntersectionBuffer, and a user
    kernel calling the header-only rb2::trace_ray; both must agree."""
    import shutil
    import subprocess
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    lib = root / "renderbox2_b200" / "_lib"
    exe = tmp_path / "compat_trace"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2", f"-I{root / 'include'}",
                    str(root / "tests" / "cpp" / "compat_trace.cu"), f"-L{lib}", "-lrb2", "-Xlinker", "-rpath",
                    "-Xlinker", str(lib), "-o", str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True, timeout=120).stdout
    f = dict(zip(out.split()[0::2], out.split()[1::2]))
    n, hits = int(f["rays"]), int(f["hits"])
    assert 0.3 * n < hits < n
    assert int(f["bad_hit"]) == 0 and int(f["bad_pos"]) == 0
    assert int(f["bad_prim"]) <= max(2, hits // 10000)   # edge ties between the two traversal orders
