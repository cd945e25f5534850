"""GPU parity of the layered materials (rb2_material_query) and of the path
tracer on scenes that use them, through the C ABI.

Bars: device material functions within single-precision rounding of the FP64
oracle (itself pinned to the reference's compiled BSDFs, test_oracle.py) for
every type and for multi-layer materials; the path tracer's and BDPT's images
converge to the FP64 host path tracer and host BDPT with the same materials
(error at the noise level both estimates should have, image means within 2-3 %),
mirror and glass layers included."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _materials():
    from renderbox2_b200.render import BsdfLayer as B
    return [
        [B("lambertian", (0.7, 0.5, 0.3))],
        [B("orennayar", (0.6, 0.6, 0.6), sigma_deg=25.0)],
        [B("microfacet", (0.9, 0.8, 0.7), exponent=30.0, fresnel="conductor")],
        [B("microfacet", (0.9, 0.9, 0.9), exponent=200.0, fresnel="dielectric", etai=1.0, etat=1.5)],
        [B("microfacet", (0.9, 0.9, 0.9), exponent=50.0, fresnel="noop")],
        [B("mirror", (0.9, 0.8, 0.9))],
        [B("glass", (1.0, 0.9, 1.0), etai=1.0, etat=1.5)],
        [B("lambertian", (0.5, 0.5, 0.5)), B("microfacet", (0.4, 0.4, 0.4), exponent=80.0, fresnel="dielectric",
                                              etai=1.0, etat=1.5)],
        [B("orennayar", (0.6, 0.3, 0.3), sigma_deg=40.0), B("mirror", (0.3, 0.3, 0.3)),
         B("glass", (0.8, 0.8, 0.8), etai=1.0, etat=1.33)],
    ]


def _close(got, want, what):
    """Single-precision agreement: rtol 3e-3 everywhere but near-singular
    Blinn lobes (high exponents at grazing angles amplify float rounding), where
    at most 0.1 % of values may differ by up to 5 %."""
    tight = np.isclose(got, want, rtol=3e-3, atol=3e-5)
    loose = np.isclose(got, want, rtol=5e-2, atol=3e-5)
    assert loose.all(), (what, np.argwhere(~loose)[:5])
    assert (~tight).mean() <= 1e-3, (what, (~tight).mean())


def test_device_materials_equal_oracle(rb, orc, cuda):
    from renderbox2_b200.render import DeviceScene, material_descs
    torch = cuda
    mats = _materials()
    room = rb.RoomScene(seed=3, n_boxes=2, n_spheres=2, sphere_subdiv=1, n_lights=1)
    n_mat = room.albedo.shape[0]
    assert n_mat >= len(mats)
    full = mats + [[mats[0][0]]] * (n_mat - len(mats))
    ds = DeviceScene(room, materials=full)
    arr = orc.materials_array(material_descs(full))
    rng = np.random.Generator(np.random.PCG64(5))
    n = 3000
    for k in range(len(mats)):
        v = rng.normal(size=(3, n, 3))
        v /= np.linalg.norm(v, axis=2, keepdims=True)
        ids = torch.full((n,), k, dtype=torch.int32, device="cuda")
        q = np.concatenate([v[0], v[1], v[2]], 1).astype(np.float32)
        got = ds.material_query(ids, torch.from_numpy(q).cuda()).cpu().numpy()
        want = orc.material_query(arr[k:k + 1], False, q.astype(np.float64))
        _close(got, want, f"eval, material {k}")
        u = rng.uniform(size=(n, 3))
        q2 = np.concatenate([v[0], v[1], u], 1).astype(np.float32)
        got = ds.material_query(ids, torch.from_numpy(q2).cuda(), sample=True).cpu().numpy()
        want = orc.material_query(arr[k:k + 1], True, q2.astype(np.float64))
        # Samples that land on a component boundary (uc * layers near an integer)
        # may pick different layers in single and double precision: skip those.
        nl = len(mats[k])
        edge = np.abs(u[:, 2] * nl - np.round(u[:, 2] * nl)) < 1e-5
        _close(got[~edge], want[~edge], f"sample, material {k}")


def _layered_room(rb):
    room = rb.RoomScene(seed=2, n_boxes=10, n_spheres=60, sphere_subdiv=2, n_lights=1, emission=10.0)
    from renderbox2_b200.render import BsdfLayer as B
    n_mat = room.albedo.shape[0]
    mats = [[B("lambertian", tuple(float(c) for c in room.albedo[m]))] for m in range(n_mat)]
    special = _materials()[1:]
    # The room's boxes and spheres (materials 6..) take the non-Lambertian materials in turn.
    for i, m in enumerate(range(6, n_mat - 1)):
        mats[m] = special[i % len(special)]
    mats[n_mat - 1] = []   # the light
    return room, mats


def test_layered_path_tracing_converges_to_host_reference(rb, orc, cuda):
    from renderbox2_b200.configs import CONFIG2 as C2
    from renderbox2_b200.render import DeviceScene, Integrator, PathIntegratorParams, material_descs
    room, mats = _layered_room(rb)
    bvh = rb.BVH(room)
    ds = DeviceScene(room, materials=mats)
    it = Integrator(rb.CudaTracer(bvh), ds)
    W, H = 96, 54
    cam = rb.PerspectiveCamera(C2["eye"], C2["lookat"], C2["up"], (W, H), C2["fov"])
    step = 4
    ii, jj = np.meshgrid(np.arange(0, W, step), np.arange(0, H, step))
    pix = (jj * W + ii).ravel()
    ref_spp = 16384
    rng = np.random.Generator(np.random.PCG64(19))
    xy = (np.repeat(np.stack([ii.ravel(), jj.ravel()], 1), ref_spp, axis=0) +
          rng.uniform(0, 1, size=(pix.size * ref_spp, 2))).astype(np.float32)
    rays = orc.ref_camera_rays(C2["eye"], C2["lookat"], C2["up"], W, H, C2["fov"], xy)
    L = orc.pt(bvh.buffers_view(), room.vertices, room.indices, room.material_ids, room.albedo, room.emission,
               room.light_ids_to_primitive_ids, rays, C2["max_depth"], C2["rr_start"], C2["rr_prob"], seed=29,
               materials=material_descs(mats)).reshape(pix.size, ref_spp, 3)
    ref = L.mean(axis=1)
    var = L.var(axis=1)                     # per-pixel variance of one sample
    assert ref.mean() > 0.0
    # Mirrors and glass make the estimator heavy-tailed, so instead of a slope
    # the error is compared with the noise both estimates should have: for an
    # unbiased renderer E[(gpu - ref)^2] = var / spp + var / ref_spp per pixel.
    ratios = {}
    for spp in (256, 4096):
        img = it.render_pt(cam, PathIntegratorParams(spp=spp, max_depth=C2["max_depth"], rr_start=C2["rr_start"],
                                                     rr_prob=C2["rr_prob"], seed=spp)).cpu().numpy()
        got = img[pix]
        mse = ((got - ref) ** 2).mean()
        expected = (var / spp + var / ref_spp).mean()
        ratios[spp] = float(mse / expected)
        if spp == 4096:
            assert abs(got.mean() / ref.mean() - 1.0) < 0.02, (got.mean(), ref.mean())
    print("layered PT error / expected noise", ratios)
    assert all(0.3 < r < 1.8 for r in ratios.values()), ratios


def _glossy_room(rb):
    """The layered room with only non-specular materials (no mirror or glass
    layer)."""
    room = rb.RoomScene(seed=2, n_boxes=10, n_spheres=60, sphere_subdiv=2, n_lights=1, emission=10.0)
    from renderbox2_b200.render import BsdfLayer as B
    n_mat = room.albedo.shape[0]
    mats = [[B("lambertian", tuple(float(c) for c in room.albedo[m]))] for m in range(n_mat)]
    special = [
        [B("orennayar", (0.6, 0.6, 0.6), sigma_deg=25.0)],
        [B("microfacet", (0.9, 0.8, 0.7), exponent=30.0, fresnel="conductor")],
        [B("microfacet", (0.9, 0.9, 0.9), exponent=40.0, fresnel="dielectric", etai=1.0, etat=1.5)],
        [B("microfacet", (0.8, 0.8, 0.8), exponent=20.0, fresnel="noop")],
        [B("lambertian", (0.5, 0.5, 0.5)), B("microfacet", (0.4, 0.4, 0.4), exponent=30.0, fresnel="dielectric",
                                              etai=1.0, etat=1.5)],
    ]
    for i, m in enumerate(range(6, n_mat - 1)):
        mats[m] = special[i % len(special)]
    mats[n_mat - 1] = []
    return room, mats


def test_layered_bdpt_converges_to_host_reference(rb, orc, cuda):
    """BDPT on glossy layered materials (Oren-Nayar, Blinn microfacet with
    each Fresnel, a two-layer material) against the FP64 host BDPT with the same
    materials: relative RMSE falls as spp^-1/2 (slope -0.5 +- 0.15), and the
    converged BDPT and path-traced images agree on their means to 3 %."""
    from renderbox2_b200.configs import CONFIG2 as C2
    from renderbox2_b200.render import (BidirectionalPathIntegratorLvcParams, DeviceScene, Integrator,
                                        PathIntegratorParams, material_descs)
    room, mats = _glossy_room(rb)
    bvh = rb.BVH(room)
    W, H, step, n_iter = 96, 54, 3, 2048
    ii, jj = np.meshgrid(np.arange(0, W, step), np.arange(0, H, step))
    pix = (jj * W + ii).ravel()
    rng = np.random.Generator(np.random.PCG64(53))
    base = np.tile(np.stack([ii.ravel(), jj.ravel()], 1), (n_iter, 1))
    xy = (base + rng.uniform(0, 1, size=base.shape)).astype(np.float32)
    rays = orc.ref_camera_rays(C2["eye"], C2["lookat"], C2["up"], W, H, C2["fov"], xy)
    ref = orc.bdpt(bvh.buffers_view(), room.vertices, room.indices, room.material_ids, room.albedo, room.emission,
                   room.light_ids_to_primitive_ids, rays, pix.size, n_iter, 2048, 6, 1, 3, 0.95, seed=59,
                   materials=material_descs(mats))
    assert ref.mean() > 0.0
    it = Integrator(rb.CudaTracer(bvh), DeviceScene(room, materials=mats))
    cam = rb.PerspectiveCamera(C2["eye"], C2["lookat"], C2["up"], (W, H), C2["fov"])
    spps, errs = [16, 64, 256], []
    for spp in spps:
        img = it.render_bdpt(cam, BidirectionalPathIntegratorLvcParams(spp=spp, max_path_length=6, connections=1,
                                                                       seed=61)).cpu().numpy()
        g = img[pix].astype(np.float64)
        assert np.isfinite(g).all() and (g >= 0).all()
        errs.append(float(np.sqrt(np.mean((g - ref) ** 2)) / ref.mean()))
    slope = np.polyfit(np.log(spps), np.log(errs), 1)[0]
    print("layered BDPT rel RMSE", dict(zip(spps, errs)), "slope", slope)
    assert errs[1] <= 0.9
    assert -0.65 <= slope <= -0.35
    cam2 = rb.PerspectiveCamera(C2["eye"], C2["lookat"], C2["up"], (160, 90), C2["fov"])
    bd = it.render_bdpt(cam2, BidirectionalPathIntegratorLvcParams(spp=512, max_path_length=6, connections=2)).cpu().numpy()
    pt = it.render_pt(cam2, PathIntegratorParams(spp=512, max_depth=4, rr_start=3, rr_prob=0.95)).cpu().numpy()
    rel = np.abs(bd.mean(0) - pt.mean(0)) / pt.mean(0)
    print("layered BDPT vs PT mean rel diff", rel)
    assert (rel < 0.03).all()


def _specular_room(rb):
    """The layered room with mirrors, glass, and materials that mix specular
    and non-specular layers.  Every material's layer colours sum below 1 per
    channel (a material picks one layer at random and scales it by the layer
    count), so no bounce gains energy and the estimators stay light-tailed."""
    room = rb.RoomScene(seed=2, n_boxes=10, n_spheres=60, sphere_subdiv=2, n_lights=1, emission=10.0)
    from renderbox2_b200.render import BsdfLayer as B
    n_mat = room.albedo.shape[0]
    mats = [[B("lambertian", tuple(float(c) for c in room.albedo[m]))] for m in range(n_mat)]
    special = [
        [B("mirror", (0.9, 0.8, 0.9))],
        [B("glass", (1.0, 0.9, 1.0), etai=1.0, etat=1.5)],
        [B("orennayar", (0.4, 0.2, 0.2), sigma_deg=40.0), B("mirror", (0.2, 0.2, 0.2)),
         B("glass", (0.3, 0.3, 0.3), etai=1.0, etat=1.33)],
        [B("lambertian", (0.5, 0.3, 0.3)), B("mirror", (0.3, 0.3, 0.3))],
        [B("microfacet", (0.9, 0.8, 0.7), exponent=30.0, fresnel="conductor")],
    ]
    for i, m in enumerate(range(6, n_mat - 1)):
        mats[m] = special[i % len(special)]
    mats[n_mat - 1] = []
    return room, mats


def test_specular_bdpt_converges_to_host_reference(rb, orc, cuda):
    """BDPT on mirrors, glass and mixed specular / non-specular materials
    against the FP64 host BDPT with the same materials.  The reference is 16
    independent host runs of 128 iterations: their mean is the image and their
    spread gives the per-sample variance, so that an unbiased renderer has a
    mean squared error of var / spp + var / 2048 per pixel; the measured error
    must lie within a factor 0.3-2 of that at 256 and 1024 spp, and the image
    means must agree to 3 %.

    The strategy weights are then checked against the path tracer: with paths
    of up to 14 segments (the path tracer at max_depth 12 covers exactly those
    up to its last vertex's NEE) the two images agree on their means to 3 %.
    At 6 segments they would differ by design: the path tracer's last vertex
    contributes only through NEE, which cannot reach a 6-segment path whose
    fifth vertex scatters specularly, while BDPT reaches it by emission.  The
    path tracer follows the reference's material_pdf, which divides by the
    non-specular layer count where material_sample_f divides by all layers; on
    these mixed materials that moves its mean by under 1 %."""
    from renderbox2_b200.configs import CONFIG2 as C2
    from renderbox2_b200.render import (BidirectionalPathIntegratorLvcParams, DeviceScene, Integrator,
                                        PathIntegratorParams, material_descs)
    room, mats = _specular_room(rb)
    bvh = rb.BVH(room)
    W, H, step, n_light = 96, 54, 3, 2048
    ii, jj = np.meshgrid(np.arange(0, W, step), np.arange(0, H, step))
    pix = (jj * W + ii).ravel()
    descs = material_descs(mats)

    def host(n_iter, seed):
        rng = np.random.Generator(np.random.PCG64(seed + 1000))
        base = np.tile(np.stack([ii.ravel(), jj.ravel()], 1), (n_iter, 1))
        xy = (base + rng.uniform(0, 1, size=base.shape)).astype(np.float32)
        rays = orc.ref_camera_rays(C2["eye"], C2["lookat"], C2["up"], W, H, C2["fov"], xy)
        return orc.bdpt(bvh.buffers_view(), room.vertices, room.indices, room.material_ids, room.albedo,
                        room.emission, room.light_ids_to_primitive_ids, rays, pix.size, n_iter, n_light, 6, 1, 3,
                        0.95, seed=seed, materials=descs)

    chunks = np.stack([host(128, 200 + c) for c in range(16)])
    ref = chunks.mean(0)
    var = 128 * chunks.var(axis=0, ddof=1)
    assert ref.mean() > 0.0
    it = Integrator(rb.CudaTracer(bvh), DeviceScene(room, materials=mats))
    cam = rb.PerspectiveCamera(C2["eye"], C2["lookat"], C2["up"], (W, H), C2["fov"])
    ratios = {}
    for spp in (256, 1024):
        img = it.render_bdpt(cam, BidirectionalPathIntegratorLvcParams(spp=spp, max_path_length=6,
                                                                       num_light_paths=n_light, connections=1,
                                                                       seed=61 + spp)).cpu().numpy()
        g = img[pix].astype(np.float64)
        assert np.isfinite(g).all() and (g >= 0).all()
        ratios[spp] = float(((g - ref) ** 2).mean() / (var / spp + var / 2048).mean())
        if spp == 1024:
            assert abs(g.mean() / ref.mean() - 1.0) < 0.03, (g.mean(), ref.mean())
    print("specular BDPT error / expected noise", ratios)
    assert all(0.3 < r < 2.0 for r in ratios.values()), ratios
    cam2 = rb.PerspectiveCamera(C2["eye"], C2["lookat"], C2["up"], (160, 90), C2["fov"])
    bd = it.render_bdpt(cam2, BidirectionalPathIntegratorLvcParams(spp=512, max_path_length=14,
                                                                   connections=2)).cpu().numpy()
    pt = it.render_pt(cam2, PathIntegratorParams(spp=512, max_depth=12, rr_start=3, rr_prob=0.95)).cpu().numpy()
    rel = np.abs(bd.mean(0) - pt.mean(0)) / pt.mean(0)
    print("specular BDPT vs PT mean rel diff (14 segments)", rel)
    assert (rel < 0.03).all()
