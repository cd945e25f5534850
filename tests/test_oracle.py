"""CPU tests of the oracle against the reference's own compiled code and the
golden fixtures, and of the rb2 builder/packer against the reference's."""
import numpy as np
import pytest

from parity import golden


def test_oracle_reproduces_golden_hits(orc):
    g = golden()
    ch, cnt = orc.trace(g["ref_nodes"], g["ref_woop"], g["ref_triidx"], g["rays"], counts=True, nthreads=1)
    assert np.array_equal(ch["prim"], g["ch_prim"])
    for k in ("t", "u", "v"):
        assert np.array_equal(ch[k].view(np.uint32), g["ch_" + k].view(np.uint32))
    assert np.array_equal(cnt["nodes"], g["ch_nodes"])
    assert np.array_equal(cnt["tris"], g["ch_tris"])
    assert np.array_equal(cnt["leafterms"], g["ch_terms"])
    ah = orc.trace(g["ref_nodes"], g["ref_woop"], g["ref_triidx"], g["rays"], any_hit=True, nthreads=1)
    assert np.array_equal(ah["prim"] >= 0, g["ah_prim"] >= 0)
    assert int((g["ch_prim"] >= 0).sum()) > 300  # fixture exercises real hits


def test_oracle_equals_bruteforce(orc):
    g = golden()
    ch = orc.trace(g["ref_nodes"], g["ref_woop"], g["ref_triidx"], g["rays"])
    bf = orc.bruteforce(g["ref_woop"], g["ref_triidx"], g["rays"])
    assert np.array_equal(ch["prim"], bf["prim"])
    assert np.array_equal(ch["t"].view(np.uint32), bf["t"].view(np.uint32))


def test_oracle_agrees_with_reference_moller_trumbore():
    g = golden()
    hit = g["ch_prim"] >= 0
    # The reference's own host triangle test (core/primitives.cu:51-70) accepts
    # every triangle the traversal reports.  Moller-Trumbore and the Woop
    # transform are different fp32 formulas for the same distance, so they
    # agree to a few ulps of the scene scale (1.0), not bit for bit.
    assert g["mt_hit"][hit].all()
    t_mt = g["mt_uvt"][hit, 2]
    t_tr = g["ch_t"][hit]
    assert np.all(np.abs(t_mt - t_tr) <= 1e-5 * np.abs(t_tr) + 4e-6)


def test_anyhit_iff_closest_hit(orc):
    g = golden()
    assert np.array_equal(g["ah_prim"] >= 0, g["ch_prim"] >= 0)


def test_reference_build_is_reproducible(orc):
    if not orc.have_ref():
        pytest.skip("reference sources not compiled here")
    g = golden()
    ref = orc.ref_build(g["vertices"], g["indices"])
    assert np.array_equal(ref["nodes"], g["ref_nodes"])
    assert np.array_equal(ref["woop"], g["ref_woop"])
    assert np.array_equal(ref["triidx"], g["ref_triidx"])


def _woop_by_tri(woop, triidx):
    w = np.asarray(woop, np.uint32).reshape(-1, 4)
    out, s = {}, 0
    while s < w.shape[0]:
        if w[s, 0] == 0x80000000:
            s += 1
            continue
        out.setdefault(int(triidx[s]), w[s:s + 3].copy())
        s += 3
    return out


def test_rb2_woop_rows_bit_equal_reference_fixture(rb):
    g = golden()
    sc = rb.Scene().add_mesh(g["vertices"], g["indices"])
    b = rb.BVH(sc)
    mine = _woop_by_tri(b.get_tri_woop_buffer(), b.get_tri_index_buffer())
    ref = _woop_by_tri(g["ref_woop"], g["ref_triidx"])
    assert set(mine) == set(ref)
    assert all(np.array_equal(mine[k], ref[k]) for k in ref)


@pytest.mark.parametrize("kind", ["heightfield", "room"])
def test_rb2_woop_rows_bit_equal_reference_builder(rb, orc, kind):
    if not orc.have_ref():
        pytest.skip("reference sources not compiled here")
    if kind == "heightfield":
        sc = rb.heightfield_scene(seed=21, grid_n=40, n_boxes=12)
    else:
        sc = rb.RoomScene(seed=22, n_boxes=6, n_spheres=12, sphere_subdiv=1)
    ref = orc.ref_build(sc.vertices, sc.indices)
    b = rb.BVH(sc)
    mine = _woop_by_tri(b.get_tri_woop_buffer(), b.get_tri_index_buffer())
    theirs = _woop_by_tri(ref["woop"], ref["triidx"])
    assert set(mine) == set(theirs)
    assert all(np.array_equal(mine[k], theirs[k]) for k in theirs)
    # SAH quality at least on par with the reference's builder.
    assert b.stats()["sah"] <= ref["sah"] * 1.05


def test_rb2_tree_gives_reference_hits(rb, orc):
    from parity import compare_closest
    g = golden()
    sc = rb.Scene().add_mesh(g["vertices"], g["indices"])
    b = rb.BVH(sc)
    mine = orc.trace(b.get_node_buffer(), b.get_tri_woop_buffer(), b.get_tri_index_buffer(), g["rays"])
    ref = {"prim": g["ch_prim"], "t": g["ch_t"], "u": g["ch_u"], "v": g["ch_v"]}
    as_dev = np.stack([mine["prim"], mine["t"].view(np.int32), mine["u"].view(np.int32), mine["v"].view(np.int32)], 1)
    ties, bad, first = compare_closest(orc, as_dev, ref, g["ref_woop"], g["ref_triidx"], g["rays"])
    assert bad == 0, f"ray {first} differs beyond a tie"


def test_camera_matrices_reproduce_reference_rays(rb):
    """Host camera set-up: applying rb2's matrices with IEEE single ops in the
    device kernel's order reproduces the reference camera's rays bit-exactly."""
    from renderbox2_b200.configs import CONFIG1 as C1
    g = golden()
    cam = rb.PerspectiveCamera(C1["eye"], C1["lookat"], C1["up"], (C1["width"], C1["height"]), C1["fov"])
    r2c = np.array(cam.c.raster_to_camera, np.float32).reshape(4, 4)
    c2w = np.array(cam.c.camera_to_world, np.float32).reshape(4, 4)
    f = np.float32

    def row(m, i, x, y, z, w):
        return ((m[i, 0] * x + m[i, 1] * y) + m[i, 2] * z) + m[i, 3] * w

    xy = g["cam_xy"]
    x, y = xy[:, 0].astype(f), xy[:, 1].astype(f)
    z0, one = np.zeros_like(x), np.ones_like(x)
    px, py, pz, pw = (row(r2c, i, x, y, z0, one) for i in range(4))
    px, py, pz = px / pw, py / pw, pz / pw
    inv = f(1.0) / np.sqrt((px * px + py * py) + pz * pz)
    dx, dy, dz = px * inv, py * inv, pz * inv
    ow = row(c2w, 3, z0, z0, z0, one)
    o = [row(c2w, i, z0, z0, z0, one) / ow for i in range(3)]
    d = [row(c2w, i, dx, dy, dz, z0) for i in range(3)]
    mine = np.stack([o[0], o[1], o[2], z0, d[0], d[1], d[2], np.full_like(x, np.finfo(f).max)], 1)
    assert np.array_equal(mine.view(np.uint32), g["cam_rays"].view(np.uint32))


def test_pcg32_matches_oracle_restatement(rb, orc):
    import ctypes as C
    L = orc.orc_lib()

    class Pcg(C.Structure):
        _fields_ = [("state", C.c_uint64), ("inc", C.c_uint64)]

    L.rb2o_pcg32_seed.argtypes = [C.POINTER(Pcg), C.c_uint64, C.c_uint64]
    L.rb2o_pcg32_next.restype = C.c_uint32
    L.rb2o_pcg32_next.argtypes = [C.POINTER(Pcg)]
    r = Pcg()
    L.rb2o_pcg32_seed(C.byref(r), 42, 54)
    ref = np.array([L.rb2o_pcg32_next(C.byref(r)) for _ in range(6)], np.uint32)
    assert np.array_equal(rb.pcg32(42, 54, 6), ref)
    # O'Neill's published demo sequence for seed 42, stream 54.
    assert ref[0] == 0xA15C02B7 and ref[1] == 0x7B47F409


def test_isect_record_matches_reference_arithmetic(rb, orc):
    """The oracle's intersection record (geometric normal, hit position) is
    bit-identical to the reference's own compute_normal and Ray::operator()
    compiled from its sources; the remaining fields are plain copies."""
    if not orc.have_ref():
        pytest.skip("reference library not built")
    scene = rb.RoomScene(seed=9, n_boxes=6, n_spheres=12, sphere_subdiv=2, n_lights=1)
    bvh = rb.BVH(scene)
    nodes, woop, tri = bvh.buffers_view()
    rays, _ = rb.surface_rays(scene, seed=10, n=3000)
    hits = orc.trace(nodes, woop, tri, rays)
    v = np.asarray(scene.vertices, np.float32).reshape(-1, 3)
    ix = np.asarray(scene.indices, np.uint32).reshape(-1, 3)
    m = np.asarray(scene.material_ids, np.uint32).reshape(-1)
    rec = orc.isect(v, np.concatenate([ix, m[:, None]], 1), rays, hits)
    hit = np.nonzero(hits["prim"] >= 0)[0]
    assert hit.size > 1000
    for i in hit:
        p = hits["prim"][i]
        ng, pt = orc.ref_normal_and_point(v[ix[p, 0]], v[ix[p, 1]], v[ix[p, 2]], rays[i], hits["t"][i])
        assert np.array_equal(ng.view(np.uint32), rec["ng"][:, i].view(np.uint32)), i
        assert np.array_equal(pt.view(np.uint32), rec["position"][:, i].view(np.uint32)), i
        assert rec["front"][i] == (1 if float(np.dot(ng.astype(np.float64), rays[i, 4:7])) < 0 else 0) or \
            abs(float(np.dot(ng.astype(np.float64), rays[i, 4:7]))) < 1e-6
        assert rec["material"][i] == m[p] and rec["prim"][i] == p
    miss = hits["prim"] < 0
    assert (rec["intersected"][miss] == 0).all() and np.isnan(rec["position"][:, miss]).all()


def _bsdf_materials():
    from renderbox2_b200.render import BsdfLayer, material_descs
    return material_descs([
        [BsdfLayer("lambertian", (0.7, 0.5, 0.3))],
        [BsdfLayer("orennayar", (0.6, 0.6, 0.6), sigma_deg=25.0)],
        [BsdfLayer("microfacet", (0.9, 0.8, 0.7), exponent=30.0, fresnel="conductor")],
        [BsdfLayer("microfacet", (0.9, 0.9, 0.9), exponent=200.0, fresnel="dielectric", etai=1.0, etat=1.5)],
        [BsdfLayer("microfacet", (0.9, 0.9, 0.9), exponent=50.0, fresnel="noop")],
        [BsdfLayer("mirror", (0.9, 0.8, 0.9))],
        [BsdfLayer("glass", (1.0, 0.9, 1.0), etai=1.0, etat=1.5)],
    ])


def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def test_material_functions_match_reference_bsdfs(orc):
    """The oracle's FP64 BSDFs agree with the reference's own material_f,
    material_pdf and material_sample_f (core/reflection.cu, core/material.cu,
    compiled in place) to single-precision rounding, for every single-layer
    material type.  One documented difference: when a Blinn microfacet sample
    reflects below the surface, the reference still returns the microfacet
    value (its sample_f skips the side test material_f applies); here f = 0."""
    if not orc.have_ref():
        pytest.skip("reference library not built")
    rng = np.random.Generator(np.random.PCG64(11))
    arr = orc.materials_array(_bsdf_materials())
    n = 1500
    for k in range(arr.shape[0]):
        N, wo, wi = _unit(rng, n), _unit(rng, n), _unit(rng, n)
        q = np.concatenate([N, wo, wi], 1)
        ours, ref = orc.material_query(arr[k:k + 1], False, q), orc.ref_material(arr[k:k + 1], False, q)
        np.testing.assert_allclose(ours, ref, rtol=5e-4, atol=1e-6, err_msg=f"eval, material {k}")
        u = rng.uniform(size=(n, 3))
        q2 = np.concatenate([N, wo, u], 1)
        ours, ref = orc.material_query(arr[k:k + 1], True, q2), orc.ref_material(arr[k:k + 1], True, q2)
        ok = ref[:, 6] > 0
        assert np.array_equal(ours[:, 6] > 0, ok) or arr[k]["layer"][0]["type"] == 4
        below = (np.einsum("ij,ij->i", ref[:, :3], N) * np.einsum("ij,ij->i", wo, N)) <= 0
        quirk = ok & below & (arr[k]["layer"][0]["type"] == 4)
        keep = ok & ~quirk
        np.testing.assert_allclose(ours[keep], ref[keep], rtol=2e-3, atol=2e-5, err_msg=f"sample, material {k}")
        assert (ours[quirk, 3:6] == 0).all()


def test_raycast_shade_rules(orc):
    """The restatement of kernel_ray_cast_update (integrators/integrator_raycast.cu:
    65-124): misses black in every mode, the palette wraps at 15, the uv mode
    is empty, a material's colour is its first layer's (the emission for an
    emitter, black for Oren-Nayar), normals are unit geometric normals."""
    from renderbox2_b200.render import BsdfLayer as B, material_descs
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1], [2, 0, 1]], np.float32)
    idx = np.array([[0, 1, 2], [0, 2, 3], [3, 4, 5], [1, 4, 5]], np.uint32)
    tri_mat = np.array([0, 1, 2, 3], np.uint32)
    albedo = np.array([[0.1, 0.2, 0.3], [0.4, 0.5, 0.6], [0.7, 0.8, 0.9], [0.2, 0.2, 0.2]], np.float32)
    emission = np.zeros((4, 3), np.float32)
    emission[3] = (5.0, 6.0, 7.0)
    mats = material_descs([[B("lambertian", (0.1, 0.2, 0.3))], [B("orennayar", (0.5, 0.5, 0.5), sigma_deg=20.0)],
                           [B("mirror", (0.9, 0.8, 0.7)), B("lambertian", (0.3, 0.3, 0.3))], []])
    prim = np.array([-1, 0, 1, 2, 3], np.int64)
    args = (v, idx, tri_mat, albedo, emission)
    for mode in range(5):
        assert not orc.raycast_shade(prim[:1], mode, *args, mats).any()
    # The palette mode reads no geometry: ids past the triangle count only index the palette.
    ids = np.array([0, 14, 15, 16, 29, 30])
    assert np.array_equal(orc.raycast_shade(ids, 0, *args), orc.RAYCAST_PALETTE[[0, 14, 0, 1, 14, 0]])
    assert not orc.raycast_shade(prim, 3, *args, mats).any()
    mat = orc.raycast_shade(np.array([0, 1, 2, 3]), 1, *args, mats)
    np.testing.assert_array_equal(mat, np.array([[0.1, 0.2, 0.3], [0, 0, 0], [0.9, 0.8, 0.7], [5, 6, 7]], np.float32))
    plain = orc.raycast_shade(np.array([0, 1, 2]), 1, *args)
    np.testing.assert_array_equal(plain, albedo[:3])
    nrm = orc.raycast_shade(np.array([0, 1, 2, 3]), 2, *args)
    np.testing.assert_allclose(np.linalg.norm(nrm, axis=1), 1.0, rtol=1e-6)
    np.testing.assert_allclose(nrm[0], (0, 0, 1))
    assert np.array_equal(orc.raycast_shade(np.array([-1, 2]), 4, *args), np.array([[0, 0, 0], [1, 1, 1]], np.float32))
    # The sample positions stay inside their pixels and are sample-major.
    xy = orc.jittered_raster(7, 3, 2, 11)
    base = np.tile(np.stack([np.arange(21) % 7, np.arange(21) // 7], 1), (2, 1))
    assert ((xy - base >= 0) & (xy - base < 1)).all()


@pytest.mark.parametrize("seed,tris", [(4000, 1_000), (4017, 40_000), (4040, 300_000)])
def test_oracle_workload_generator_equals_product_generator(rb, orc, seed, tris):
    """The CPU reference arm builds the batching workload without the product
    library; its generator must give the product's scenes and rays bit for bit."""
    sc = rb.heightfield_for_triangles(seed=seed, n_tris=tris)
    v, i = orc.gen_heightfield_for_triangles(seed, tris)
    assert np.array_equal(v.view(np.uint32), sc.vertices.view(np.uint32))
    assert np.array_equal(i, sc.indices)
    r1, f1 = rb.surface_rays(sc, seed=seed + 500, n=150_000)
    r2, f2 = orc.gen_surface_rays(v, i, seed + 500, 150_000)
    assert np.array_equal(r1.view(np.uint32), r2.view(np.uint32))
    assert np.array_equal(f1, f2)


def test_tie_scene_produces_ties_on_both_trees(rb, orc):
    """Rays through shared edges and vertices of dyadic geometry: most are
    accepted by 2-6 triangles at the same t; the traversal's pick is one of
    them; the BVH-walking tie count never exceeds the exhaustive one."""
    from tie_scene import tie_rays, tie_scene
    scene = tie_scene(rb)
    rays, kinds = tie_rays()
    bvh = rb.BVH(scene)  # buffers_view() borrows the BVH's memory: keep it alive
    trees = [bvh.buffers_view()]
    if orc.have_ref():
        r = orc.ref_build(scene.vertices, scene.indices)
        trees.append((r["nodes"], r["woop"], r["triidx"]))
    for nodes, woop, tri in trees:
        h = orc.trace(nodes, woop, tri, rays)
        assert (h["prim"] >= 0).all()
        exact = orc.tie_count(woop, tri, rays, h)
        walked = orc.tie_count(woop, tri, rays, h, nodes=nodes)
        assert (exact >= 1).all(), "the reported triangle must accept at its own t"
        assert (walked <= exact).all()
        assert (exact >= 2).mean() > 0.5
        for k in ("vertex", "edge", "diagonal", "box_edge", "box_corner"):
            assert (exact[kinds == k] >= 2).any(), k
        # The exhaustive search agrees with the traversal on t, except where
        # an axis-parallel ray runs exactly in a box's boundary plane: the
        # slab test (zero direction replaced by +-2^-80) culls that box, as
        # the reference's traversal does, so the traversal's t is larger.
        bf = orc.bruteforce(woop, tri, rays)
        assert (h["t"] >= bf["t"]).all()
        assert (h["t"] == bf["t"]).mean() > 0.99


def test_compat_formulas_pinned_to_the_reference(orc):
    """The two reference formulas the compatibility modes restate, against the
    reference's compiled functions: the AO direction of
    cosine_sample_hemisphere_normal (core/montecarlo.cu:133-151; NaN exactly
    where the oracle reports it undefined) and DiffuseAreaLight::Le's
    direction and Le / pdf (core/lights.cu:63-69), whose pdf uses the
    reference's triangle area of 0.5."""
    if not orc.have_ref():
        pytest.skip("oracle/_ref not built")
    rng = np.random.Generator(np.random.PCG64(8))
    normals = list(rng.normal(size=(200, 3))) + [np.array(v, float) for v in
                                                 ((0, 1, 0), (0, -1, 0), (1, 0, 0), (-1, 0, 0), (0, 0, 1), (0, 0, -1))]
    undefined = 0
    for n in normals:
        n = np.asarray(n, np.float32)
        n = (n / np.sqrt(np.dot(n, n))).astype(np.float32)
        for u1, u2 in rng.uniform(0, 1, size=(8, 2)).astype(np.float32):
            ref = orc.ref_ao_direction(n, u1, u2)
            got = orc.ao_ref_dir(n.astype(np.float64), float(u1), float(u2))
            if got is None:
                undefined += 1
                assert np.isnan(ref).any()
            else:
                assert np.allclose(got, ref, atol=2e-6), (n, u1, u2, got, ref)
    assert undefined > 0  # normals along +-z have no X axis there
    v0, v1, v2 = np.array([0.2, 1.0, 0.1]), np.array([0.6, 1.0, 0.1]), np.array([0.2, 1.0, 0.5])
    emit = np.array([10.0, 10.0, 10.0])
    ln = np.cross(v1 - v0, v2 - v0)
    area = 0.5 * np.linalg.norm(ln)
    ln = ln / np.linalg.norm(ln)
    # The reference's compute_area (core/primitives.h:273-276) halves the length
    # of the already normalized normal: every triangle has area 0.5 in its pdfs.
    assert abs(area - 0.08) < 1e-12
    lit = 0
    for u in rng.uniform(0, 1, size=(400, 4)).astype(np.float32):
        _, d_ref, pdf, L = orc.ref_light_le(v0, v1, v2, emit, u)
        d, k = orc.light_le_ref(ln, 0.5, float(u[2]), float(u[3]))
        assert np.allclose(d, d_ref, atol=2e-6)
        contrib = L[0] / pdf if pdf > 0 else 0.0
        assert np.isclose(emit[0] * k, contrib, rtol=1e-5, atol=1e-6), (u, k, L, pdf)
        lit += k > 0
    assert 0 < lit < 400  # only directions toward the light's front carry Le
