"""CPU tests of the compressed 8-wide layout (RB2_NODE_ORDER_CW8) that the
tracer collapses from the binary Compact2 tree: every triangle reference of
the binary leaves is present exactly once, node indices and triangle ranges
are in bounds, and the leaf holding the oracle's closest hit is reachable: the
hit point lies inside the leaf's quantized box and every ancestor's, so the
conservative box tests of the wide traversal cannot miss it."""
import collections

import numpy as np
import pytest


def _decode(nodes):
    n = nodes.shape[0]
    b = nodes.view(np.uint8).reshape(n, 80)
    p = nodes[:, 0:3].view(np.float32).astype(np.float64)
    scale = np.ldexp(1.0, b[:, 12:15].astype(np.int32) - 127)
    imask = b[:, 15].astype(np.uint32)
    child_base = nodes[:, 4].astype(np.int64)
    tri_base = nodes[:, 5].astype(np.int64)
    tmask = nodes[:, 6].astype(np.uint32)
    q = {}
    for a, (lo, hi) in enumerate(((32, 40), (48, 56), (64, 72))):
        q[("lo", a)] = b[:, lo:lo + 8].astype(np.float64)
        q[("hi", a)] = b[:, hi:hi + 8].astype(np.float64)
    lo = np.stack([p[:, a:a + 1] + q[("lo", a)] * scale[:, a:a + 1] for a in range(3)], -1)  # (n, 8, 3)
    hi = np.stack([p[:, a:a + 1] + q[("hi", a)] * scale[:, a:a + 1] for a in range(3)], -1)
    return imask, child_base, tri_base, tmask, lo, hi


def _binary_leaf_refs(bvh):
    nodes, woop, tri = bvh.buffers_view()
    refs = []
    for w in nodes.reshape(-1, 16)[:, 12:14].view(np.int32).ravel():
        if w < 0:
            k = ~int(w)
            while woop[k, 0] != 0x80000000:
                refs.append(int(tri[k]))
                k += 3
    return refs


def _degenerate_scene(rb):
    """300 coincident triangles (no split separates them, so the SBVH's
    leaves hold hundreds of refs: the layout's ref-list nodes) among 50 small
    scattered ones."""
    rng = np.random.Generator(np.random.PCG64(1))
    v, idx = [], []
    for _ in range(300):
        b = len(v)
        v += [(0, 0, 0), (1, 0, 0), (0, 1, 0)]
        idx.append((b, b + 1, b + 2))
    for _ in range(50):
        c = rng.uniform(-2, 2, 3)
        b = len(v)
        v += [tuple(c), tuple(c + rng.uniform(0, .2, 3)), tuple(c + rng.uniform(0, .2, 3))]
        idx.append((b, b + 1, b + 2))
    return rb.Scene().add_mesh(np.array(v, np.float32), np.array(idx, np.uint32))


def _rays_at_cluster(n, seed):
    """Rays from above and below the unit triangle toward points inside it."""
    rng = np.random.Generator(np.random.PCG64(seed))
    o = rng.uniform(-1.0, 2.0, (n, 3))
    o[:, 2] = np.where(rng.uniform(size=n) < 0.5, 2.0, -2.0)
    u = rng.uniform(size=(n, 2))
    u = np.where(u.sum(1, keepdims=True) > 1, 1 - u, u)
    tgt = np.stack([u[:, 0], u[:, 1], np.zeros(n)], 1)
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, :3], r[:, 4:7], r[:, 7] = o, d, 3.0e38
    return r


def test_cw8_layout_on_a_room(rb, orc):
    """The config-2 style room: axis-aligned walls and boxes (flat leaf boxes)
    and icospheres."""
    sc = rb.RoomScene(seed=4, n_boxes=12, n_spheres=40, sphere_subdiv=2, n_lights=2)
    r, _ = rb.surface_rays(sc, seed=9, n=3000)
    _check_layout(rb, orc, rb.BVH(sc), r)


def test_cw8_layout_splits_large_leaves(rb, orc):
    bvh = rb.BVH(_degenerate_scene(rb))
    _check_layout(rb, orc, bvh, _rays_at_cluster(2000, 5))


@pytest.mark.parametrize("seed,n_tris,n_boxes", [(3, 2_000, 4), (8, 40_000, 30)])
def test_cw8_layout_is_complete_and_conservative(rb, orc, seed, n_tris, n_boxes):
    sc = rb.heightfield_for_triangles(seed=seed, n_tris=n_tris, n_boxes=n_boxes)
    r, _ = rb.surface_rays(sc, seed=seed + 1, n=3000)
    _check_layout(rb, orc, rb.BVH(sc), r)


def _check_layout(rb, orc, bvh, r):
    cw = bvh.cw8_layout()
    nodes, triidx = cw["nodes"], cw["triidx"]
    n, nt = nodes.shape[0], triidx.shape[0]
    assert 1 <= cw["depth"] <= 72
    assert collections.Counter(triidx.tolist()) == collections.Counter(_binary_leaf_refs(bvh))
    # Woop rows are the binary layout's rows of the same references.
    nodes_b, woop_b, tri_b = bvh.buffers_view()
    rows_b = collections.defaultdict(set)
    for w in nodes_b.reshape(-1, 16)[:, 12:14].view(np.int32).ravel():
        if w < 0:
            k = ~int(w)
            while woop_b[k, 0] != 0x80000000:
                rows_b[int(tri_b[k])].add(woop_b[k:k + 3].tobytes())
                k += 3
    for i in range(nt):
        assert cw["woop"][i].tobytes() in rows_b[int(triidx[i])]
    imask, child_base, tri_base, tmask, lo, hi = _decode(nodes)
    parent = {}
    tri_loc = collections.defaultdict(list)
    assert (nodes[:, 7] == 0).all() and (tmask < (1 << 24)).all()
    for i in range(n):
        for s in range(8):
            bits = (int(tmask[i]) >> (3 * s)) & 7
            if (imask[i] >> s) & 1:
                assert bits == 0
                c = int(child_base[i]) + bin(int(imask[i]) & ((1 << s) - 1)).count("1")
                assert 0 < c < n and c not in parent
                parent[c] = (i, s)
            elif bits:
                assert bits in (1, 3, 7)
                off = bin(int(tmask[i]) & ((1 << (3 * s)) - 1)).count("1")
                cnt = bits.bit_length()
                assert int(tri_base[i]) + off + cnt <= nt
                for k in range(cnt):
                    tri_loc[int(triidx[int(tri_base[i]) + off + k])].append((i, s))
    assert len(parent) == n - 1          # a tree: every node but the root has one parent
    # Reachability of the oracle's closest hits.
    want = orc.trace(*bvh.buffers_view(), r)
    hit = np.nonzero(want["prim"] >= 0)[0]
    assert hit.size > 100
    for k in hit:
        P = r[k, :3].astype(np.float64) + float(want["t"][k]) * r[k, 4:7].astype(np.float64)
        ok = False
        for node, s in tri_loc[int(want["prim"][k])]:
            inside = True
            while True:
                if not ((lo[node, s] <= P).all() and (P <= hi[node, s]).all()):
                    inside = False
                    break
                if node == 0:
                    break
                node, s = parent[node]
            if inside:
                ok = True
                break
        assert ok, f"ray {k}: hit point outside every chain of boxes of triangle {want['prim'][k]}"
