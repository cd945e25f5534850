"""GPU test of rb2_trace_batch_noalloc, the batched trace for callers that
cannot let a library allocate device memory (hosts that own all device memory
through their own arena or a fixed budget, and loops where cudaMalloc/cudaFree
must not appear).

The caller owns every buffer: here the BVH, rays and outputs live in torch
tensors allocated by the test, and the library uses only its fixed
file-scope scratch array.  Results must equal the regular batched entry point
(rb2_batch_create / rb2_batch_launch) bit for bit and the CPU oracle, on two
calls in a row (the scratch array keeps the previous call's contents, so the
second call checks that it is cleared correctly), and the guard-bit query
(rb2_trace_batch_noalloc_status) must read 0 after each.  Collected last on
purpose."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


class NoAllocJob(C.Structure):
    _fields_ = [("d_nodes", C.c_void_p), ("d_woop", C.c_void_p), ("d_triidx", C.c_void_p), ("d_rays", C.c_void_p),
                ("n", C.c_uint64), ("mode", C.c_uint32), ("reserved", C.c_uint32), ("d_mask", C.c_void_p),
                ("d_out", C.c_void_p)]


def _bind(rb):
    fn = rb.lib().rb2_trace_batch_noalloc
    fn.argtypes = [C.POINTER(NoAllocJob), C.c_uint32, C.c_void_p]
    fn.restype = C.c_int
    return fn


def _status(rb, stream):
    """Guard bits of the last call, read through rb2_trace_batch_noalloc_status."""
    fn = rb.lib().rb2_trace_batch_noalloc_status
    fn.argtypes = [C.POINTER(C.c_uint32), C.c_void_p]
    fn.restype = C.c_int
    word = C.c_uint32(0xFFFFFFFF)
    assert fn(C.byref(word), stream) == 0, rb.lib().rb2_last_error()
    return word.value


def _caller_owned_bvh(torch, bvh):
    """Uploads a BVH into tensors the caller owns (Woop rows + 2 spare uint4)."""
    nodes, woop, tri = bvh.buffers_view()
    d_nodes = torch.from_numpy(nodes.view(np.int32).copy()).cuda()
    w = np.zeros((woop.shape[0] + 2, 4), np.uint32)
    w[: woop.shape[0]] = woop
    d_woop = torch.from_numpy(w.view(np.int32)).cuda()
    d_tri = torch.from_numpy(tri.view(np.int32).copy()).cuda()
    return d_nodes, d_woop, d_tri


def _out_like(torch, n, mode):
    if mode == 2:
        return torch.full((n,), 9, dtype=torch.uint8, device="cuda")
    return torch.full((n, 4), 9, dtype=torch.int32, device="cuda")


def test_noalloc_matches_batched_entry_point_twice(rb, orc, cuda):
    torch = cuda
    fn = _bind(rb)
    specs = [(3_000, 40_000, rb.MODE_CLOSEST), (80_000, 100_000, rb.MODE_OCCLUSION), (500, 7, rb.MODE_ANY),
             (20_000, 65_536, rb.MODE_CLOSEST)]
    keep, ref_jobs, ref_outs, host_rays = [], [], [], []
    na = (NoAllocJob * len(specs))()
    for k, (tris, n, mode) in enumerate(specs):
        sc = rb.heightfield_for_triangles(seed=600 + k, n_tris=tris, n_boxes=4)
        bvh = rb.BVH(sc)
        tr = rb.CudaTracer(bvh)
        r, _ = rb.surface_rays(sc, seed=650 + k, n=n)
        r[::2, 4:7] *= -1.0
        d_rays = torch.from_numpy(r).cuda()
        host_rays.append(r)
        ref_out = _out_like(torch, n, mode)
        ref_jobs.append((tr, d_rays, mode, ref_out, None))
        ref_outs.append(ref_out)
        d_nodes, d_woop, d_tri = _caller_owned_bvh(torch, bvh)
        keep.append((bvh, tr, d_rays, d_nodes, d_woop, d_tri))
        na[k].d_nodes = d_nodes.data_ptr()
        na[k].d_woop = d_woop.data_ptr()
        na[k].d_triidx = d_tri.data_ptr()
        na[k].d_rays = d_rays.data_ptr()
        na[k].n = n
        na[k].mode = mode
        na[k].d_mask = None
    batch = rb.TraceBatch(ref_jobs)
    batch.launch()
    torch.cuda.synchronize()
    assert batch.status() == 0

    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        outs = [_out_like(torch, spec[1], spec[2]) for spec in specs]
        for k, o in enumerate(outs):
            na[k].d_out = o.data_ptr()
        rc = fn(na, len(specs), stream)
        assert rc == 0, rb.lib().rb2_last_error()
        assert _status(rb, stream) == 0, "guard bits set by a no-alloc call"
        torch.cuda.synchronize()
        for k, (o, ref) in enumerate(zip(outs, ref_outs)):
            assert torch.equal(o, ref), f"call {call}, job {k} differs from rb2_batch_launch"
        # and directly against the CPU oracle on the same buffers
        for k, ((tris, n, mode), o) in enumerate(zip(specs, outs)):
            nodes, woop, tri = keep[k][0].buffers_view()
            want = orc.trace(nodes, woop, tri, host_rays[k], any_hit=(mode != rb.MODE_CLOSEST))
            got = o.cpu().numpy()
            if mode == rb.MODE_OCCLUSION:
                assert np.array_equal(got.astype(bool), want["prim"] >= 0), f"call {call}, job {k}"
            elif mode == rb.MODE_ANY:
                assert np.array_equal(got[:, 0] >= 0, want["prim"] >= 0), f"call {call}, job {k}"
            else:
                assert np.array_equal(got[:, 0], want["prim"]), f"call {call}, job {k}"
                assert np.array_equal(got[:, 1].view(np.uint32), want["t"].view(np.uint32)), f"call {call}, job {k}"
    # closest-hit job sanity: real hits were produced
    assert (ref_outs[0][:, 0] >= 0).float().mean().item() > 0.3


def test_noalloc_rejects_oversized_batches(rb, cuda):
    fn = _bind(rb)
    too_many = 257  # RB2_NOALLOC_MAX_JOBS + 1
    jobs = (NoAllocJob * too_many)()
    rc = fn(jobs, too_many, None)
    assert rc == 1  # RB2_EINVAL
    msg = rb.lib().rb2_last_error().decode()
    assert "exceed" in msg and "256" in msg
    assert fn(jobs, 0, None) == 0  # an empty batch is a no-op
