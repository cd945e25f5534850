"""Ties at shared edges and vertices, on the GPU, for every node layout.

The rays of tests/tie_scene.py hit lattice vertices, edge and diagonal
midpoints of a flat dyadic grid and the edges and corners of dyadic boxes, so
two to six triangles accept each of most rays at exactly the same t (counted
by the oracle over every triangle).  The reference's rule is
`tmin < t < hitT` (accelerators/sbvh/kepler_dynamic_fetch.h:264): the first
triangle tested keeps the hit.

* Binary layouts (the reference-built tree and rb2's tree in DFS or BFS node
  order) test triangles in the oracle's order, so prim, t, u and v must equal
  the oracle's bit for bit on every ray, ties included.
* The 4-wide and compressed 8-wide layouts test the same triangles in another
  order, so at a tie they may report the other triangle: allowed only when
  the oracle confirms both accept at the same t, and counted.  The vertical
  and axis-parallel rays of this scene also meet a second, measure-zero case:
  a ray with a direction component exactly 0 that runs exactly in a binary
  box's boundary plane is culled by the reference's slab test (the zero is
  replaced by +-2^-80, so the slab there is [0, 0] or empty), and the
  reference misses the nearest triangle in that box.  The compressed 8-wide
  boxes are widened, so that layout reports the true nearest hit there (its t
  equals the exhaustive search's); those rays are counted as
  reference-culled.  The 4-wide layout keeps the exact binary boxes and the
  binary slab arithmetic, so it culls them as the reference does.
* Any-hit and occlusion decisions must agree everywhere, except that an
  any-hit ray the reference culls may be occluded in the 8-wide layout."""
import numpy as np
import pytest

from parity import compare_closest_wide
from tie_scene import tie_rays, tie_scene

pytestmark = pytest.mark.gpu

LAYOUTS = [("reference", 0), ("rb2", 0), ("rb2", 1), ("rb2", 2), ("rb2", 3)]


def _bits(h):
    h = np.asarray(h)
    return h[:, 0], h[:, 1].view(np.uint32), h[:, 2].view(np.uint32), h[:, 3].view(np.uint32)


def _setup(rb, orc, tree):
    scene = tie_scene(rb)
    if tree == "reference":
        if not orc.have_ref():
            pytest.skip("oracle/_ref not built")
        r = orc.ref_build(scene.vertices, scene.indices)
        bvh = rb.BVH.from_buffers(r["nodes"], r["woop"], r["triidx"])
    else:
        bvh = rb.BVH(scene)
    return scene, bvh


@pytest.mark.parametrize("tree,order", LAYOUTS)
def test_ties_follow_the_reference_rule(rb, orc, cuda, tree, order):
    torch = cuda
    scene, bvh = _setup(rb, orc, tree)
    nodes, woop, tri = bvh.buffers_view()
    rays, kinds = tie_rays()
    want = orc.trace(nodes, woop, tri, rays)
    n_accept = orc.tie_count(woop, tri, rays, want)
    tied = n_accept >= 2
    assert (want["prim"] >= 0).all()
    assert tied.sum() > 0.5 * rays.shape[0], "the tie scene no longer produces ties"

    tr = rb.CudaTracer(bvh)
    tr.set_node_order(order)
    d = torch.from_numpy(rays).cuda()
    got = tr.trace(d).cpu().numpy()
    if order in (0, 1):
        gp, gt, gu, gv = _bits(got)
        assert np.array_equal(gp, want["prim"])
        assert np.array_equal(gt, want["t"].view(np.uint32))
        assert np.array_equal(gu, want["u"].view(np.uint32))
        assert np.array_equal(gv, want["v"].view(np.uint32))
        divergent = 0
        culled = 0
    else:
        want_d = {"prim": want["prim"], "t": want["t"], "u": want["u"], "v": want["v"]}
        divergent, culled, bad, first = compare_closest_wide(orc, got, want_d, woop, tri, rays)
        assert bad == 0, f"ray {first} ({kinds[first]}): gpu {got[first]} vs oracle {want[first]}"
        assert divergent <= tied.sum()
        if order == 2:
            assert culled == 0, "the 4-wide layout keeps the binary boxes: it must cull as the reference does"
    want_ah = orc.trace(nodes, woop, tri, rays, any_hit=True)
    got_ah = tr.trace(d, any_hit=True).cpu().numpy()
    got_occ = tr.trace_occlusion(d).cpu().numpy().astype(bool)
    diff_ah = np.nonzero((got_ah[:, 0] >= 0) != (want_ah["prim"] >= 0))[0]
    diff_occ = np.nonzero(got_occ != (want_ah["prim"] >= 0))[0]
    if order == 3:
        # Only rays the reference culls may differ, and only toward occluded.
        axis_parallel = (rays[:, 4:7] == 0.0).any(axis=1)
        for diff in (diff_ah, diff_occ):
            assert axis_parallel[diff].all() and (want_ah["prim"][diff] < 0).all()
    else:
        assert diff_ah.size == 0 and diff_occ.size == 0
    assert tr.status() == 0
    per_kind = {k: int(tied[kinds == k].sum()) for k in np.unique(kinds)}
    print(f"{tree} order {order}: {int(tied.sum())} tied rays of {rays.shape[0]} {per_kind}; "
          f"GPU chose the other triangle of a confirmed tie on {divergent}; reference-culled rays {culled}")


@pytest.mark.parametrize("order,reorder", [(0, 0), (3, 0), (1, 4), (0, 5)])
def test_ties_in_the_batched_launch(rb, orc, cuda, order, reorder):
    """The job-table launch (closest hit + occlusion jobs) on the tie rays,
    with and without ray reordering (which changes only which rays share a
    warp, so the binary layouts stay bit-identical at every tie)."""
    torch = cuda
    scene, bvh = _setup(rb, orc, "rb2")
    nodes, woop, tri = bvh.buffers_view()
    rays, _ = tie_rays()
    want = orc.trace(nodes, woop, tri, rays)
    tr = rb.CudaTracer(bvh)
    d = torch.from_numpy(rays).cuda()
    out_h = torch.full((rays.shape[0], 4), 7, dtype=torch.int32, device="cuda")
    out_o = torch.full((rays.shape[0],), 7, dtype=torch.uint8, device="cuda")
    batch = rb.TraceBatch([(tr, d, rb.MODE_CLOSEST, out_h, None), (tr, d, rb.MODE_OCCLUSION, out_o, None)])
    batch.set_config(node_order=order, reorder=reorder)
    batch.launch()
    got = out_h.cpu().numpy()
    if order in (0, 1):
        assert np.array_equal(got[:, 0], want["prim"])
        assert np.array_equal(got[:, 1].view(np.uint32), want["t"].view(np.uint32))
        assert np.array_equal(out_o.cpu().numpy().astype(bool), want["prim"] >= 0)
    else:
        want_d = {"prim": want["prim"], "t": want["t"], "u": want["u"], "v": want["v"]}
        _, _, bad, first = compare_closest_wide(orc, got, want_d, woop, tri, rays)
        assert bad == 0, f"ray {first}"
        occ = out_o.cpu().numpy().astype(bool)
        diff = np.nonzero(occ != (want["prim"] >= 0))[0]
        assert (rays[diff, 4:7] == 0.0).any(axis=1).all()
    assert batch.status() == 0
    batch.set_config(node_order=0)


def test_ties_in_the_per_thread_trace(rb, orc, cuda):
    """The header-only per-thread trace_ray on the tie rays: bit-identical."""
    torch = cuda
    scene, bvh = _setup(rb, orc, "rb2")
    nodes, woop, tri = bvh.buffers_view()
    rays, _ = tie_rays()
    want = orc.trace(nodes, woop, tri, rays)
    tr = rb.CudaTracer(bvh)
    got = tr.trace_per_thread(torch.from_numpy(rays).cuda()).cpu().numpy()
    gp, gt, gu, gv = _bits(got)
    assert np.array_equal(gp, want["prim"])
    assert np.array_equal(gt, want["t"].view(np.uint32))
    assert np.array_equal(gu, want["u"].view(np.uint32)) and np.array_equal(gv, want["v"].view(np.uint32))
