"""GPU parity of the ray-cast integrator (rb2_render_raycast) through the C ABI.

The oracle side rebuilds the device's jittered sample positions
(oracle.jittered_raster), turns them into rays with the reference's own camera
(compiled in place), traces them with the CPU traversal, shades every sample
with the restatement of kernel_ray_cast_update (oracle.raycast_shade) and
averages in float32 in sample order, as the device does.  Bar: bit-identical
images for every shade mode but the normals, which the device normalizes with
a reciprocal square root (within 2e-6); bit-identical across wave sizes; with
a film filter, equal to the oracle's splat of the same samples."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scene(rb):
    from renderbox2_b200.render import BsdfLayer as B
    room = rb.RoomScene(seed=4, n_boxes=8, n_spheres=24, sphere_subdiv=1, n_lights=1, emission=10.0)
    n_mat = room.albedo.shape[0]
    special = [
        [B("orennayar", (0.6, 0.6, 0.6), sigma_deg=25.0)],
        [B("mirror", (0.9, 0.8, 0.9))],
        [B("glass", (1.0, 0.9, 1.0), etai=1.0, etat=1.5)],
        [B("microfacet", (0.9, 0.8, 0.7), exponent=30.0, fresnel="conductor")],
        [B("lambertian", (0.5, 0.4, 0.3)), B("mirror", (0.3, 0.3, 0.3))],
    ]
    mats = [[B("lambertian", tuple(float(c) for c in room.albedo[m]))] for m in range(n_mat)]
    for i, m in enumerate(range(6, n_mat - 1)):
        mats[m] = special[i % len(special)]
    mats[n_mat - 1] = []
    return room, mats


def _expected(orc, scene, albedo, emission, bvh, mats, W, H, spp, seed, mode, cfg=None):
    from renderbox2_b200.configs import CONFIG2
    from renderbox2_b200.render import material_descs
    c = CONFIG2 if cfg is None else cfg
    npix = W * H
    xy = orc.jittered_raster(W, H, spp, seed)
    rays = orc.ref_camera_rays(c["eye"], c["lookat"], c["up"], W, H, c["fov"], xy)
    hits = orc.trace(bvh.get_node_buffer(), bvh.get_tri_woop_buffer(), bvh.get_tri_index_buffer(), rays)
    col = orc.raycast_shade(hits["prim"], mode, scene.vertices, scene.indices, scene.material_ids, albedo, emission,
                            None if mats is None else material_descs(mats))
    acc = np.zeros((npix, 3), np.float32)
    for s in range(spp):
        acc += col[s * npix:(s + 1) * npix]
    return acc * (np.float32(1.0) / np.float32(spp)), xy, col, hits


@pytest.mark.parametrize("shade,mode", [("primitive_id", 0), ("material_id", 1), ("normals", 2), ("uvs", 3),
                                        ("uniform", 4)])
def test_raycast_equals_oracle(rb, orc, cuda, shade, mode):
    from renderbox2_b200.configs import CONFIG2 as C2
    from renderbox2_b200.render import DeviceScene, Integrator, RayCastIntegratorParams
    room, mats = _scene(rb)
    bvh = rb.BVH(room)
    it = Integrator(rb.CudaTracer(bvh), DeviceScene(room, materials=mats))
    W, H, spp, seed = 96, 54, 3, 9
    cam = rb.PerspectiveCamera(C2["eye"], C2["lookat"], C2["up"], (W, H), C2["fov"])
    want, _, _, hits = _expected(orc, room, room.albedo, room.emission, bvh, mats, W, H, spp, seed, mode)
    assert (hits["prim"] >= 0).mean() > 0.9
    got = it.render_raycast(cam, RayCastIntegratorParams(shade, spp, seed)).cpu().numpy()
    if mode == 2:
        np.testing.assert_allclose(got, want, rtol=0, atol=2e-6)
    else:
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    if mode == 3:
        assert not got.any()
    assert it.stats()["primary_rays"] == W * H * spp


def test_raycast_plain_scene_misses_and_waves(rb, orc, cuda):
    """An open heightfield seen from the config-1 pose (about 40 % of the
    samples miss) with plain albedo materials: material colours come from the
    albedo, misses are black, and several waves give the image of one."""
    from renderbox2_b200.configs import CONFIG1 as C1
    from renderbox2_b200.render import DeviceScene, Integrator, RayCastIntegratorParams
    sc = rb.heightfield_scene(seed=3, grid_n=32, n_boxes=8)
    n_mat = int(sc.material_ids.max()) + 1
    albedo = np.tile(np.array([[0.3, 0.6, 0.9]], np.float32), (n_mat, 1))
    emission = np.zeros((n_mat, 3), np.float32)
    bvh = rb.BVH(sc)
    it = Integrator(rb.CudaTracer(bvh), DeviceScene(sc, albedo=albedo, emission=emission))
    W, H, spp, seed = 80, 45, 5, 21
    cam = rb.PerspectiveCamera(C1["eye"], C1["lookat"], C1["up"], (W, H), C1["fov"])
    want, _, _, hits = _expected(orc, sc, albedo, emission, bvh, None, W, H, spp, seed, 1, C1)
    assert 0.2 < (hits["prim"] < 0).mean() < 0.8
    one = it.render_raycast(cam, RayCastIntegratorParams("material_id", spp, seed)).cpu().numpy()
    assert np.array_equal(one.view(np.uint32), want.view(np.uint32))
    assert (one == 0).all(axis=1).any()
    it.set_wave(2 * W * H)          # waves of 2, 2 and 1 samples per pixel
    waves = it.render_raycast(cam, RayCastIntegratorParams("material_id", spp, seed)).cpu().numpy()
    it.set_wave(0)
    assert np.array_equal(one.view(np.uint32), waves.view(np.uint32))
    with pytest.raises(rb.Rb2Error, match="shade"):
        it.render_raycast(cam, RayCastIntegratorParams(7, 1, seed))


def test_filtered_raycast_equals_oracle_splat(rb, orc, cuda):
    from renderbox2_b200.configs import CONFIG2 as C2
    from renderbox2_b200.render import DeviceScene, Filter, Integrator, RayCastIntegratorParams
    room, mats = _scene(rb)
    bvh = rb.BVH(room)
    it = Integrator(rb.CudaTracer(bvh), DeviceScene(room, materials=mats))
    W, H, spp, seed = 64, 36, 4, 3
    cam = rb.PerspectiveCamera(C2["eye"], C2["lookat"], C2["up"], (W, H), C2["fov"])
    _, xy, col, _ = _expected(orc, room, room.albedo, room.emission, bvh, mats, W, H, spp, seed, 0)
    L4 = np.concatenate([col, np.zeros((col.shape[0], 1), np.float32)], 1)
    it.set_filter(Filter("gaussian", 2.0, 2.0, 2.0))
    got = it.render_raycast(cam, RayCastIntegratorParams("primitive_id", spp, seed)).cpu().numpy()
    it.set_filter(None)
    want = orc.film("gaussian", 2.0, 2.0, 2.0, W, H, spp, xy, L4)
    np.testing.assert_allclose(got, want, rtol=2e-6, atol=1e-7)
