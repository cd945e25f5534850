"""GPU integrators against converged FP64 host references (the oracle's
restatement of the same estimator, run at high sample counts).

Bars (stated here, checked below):
  AO (config 1 scene and camera): RMSE within 15 % of the binomial sampling
  error sqrt(mean(p(1-p))/S) of an unbiased estimate, at S = 4, 16, 64;
  PT (room scene, config 2 camera): relative RMSE <= 0.25 at 64 spp;
  BDPT (same scene, config 3 settings): relative RMSE <= 0.8 at 64 spp, and
  its converged image mean equals the path tracer's (paths <= 6 segments);
  for all, log(RMSE) vs log(samples) has slope -0.5 +- 0.15 (error shrinks
  as 1/sqrt(samples), i.e. no bias);
  relative RMSE = sqrt(mean((gpu - ref)^2)) / mean(ref) over the sampled pixels.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _slope(samples, errs):
    return float(np.polyfit(np.log(samples), np.log(errs), 1)[0])


def test_ao_converges_to_host_reference(rb, orc, cuda):
    from renderbox2_b200.configs import CONFIG1 as C1
    from renderbox2_b200.render import AmbientOcclusionIntegratorParams, DeviceScene, Integrator
    scene = rb.heightfield_scene(seed=C1["seed"], grid_n=C1["grid_n"], n_boxes=C1["n_boxes"])
    bvh = rb.BVH(scene)
    it = Integrator(rb.CudaTracer(bvh), DeviceScene(scene))
    cam = rb.PerspectiveCamera(C1["eye"], C1["lookat"], C1["up"], (C1["width"], C1["height"]), C1["fov"])
    step = 16
    ii, jj = np.meshgrid(np.arange(0, 512, step), np.arange(0, 512, step))
    pix = (jj * 512 + ii).ravel()
    xy = np.stack([ii.ravel() + 0.5, jj.ravel() + 0.5], 1).astype(np.float32)
    prim = orc.ref_camera_rays(C1["eye"], C1["lookat"], C1["up"], 512, 512, C1["fov"], xy)
    ref = orc.ao(bvh.buffers_view(), scene.vertices, scene.indices, prim, 8192, C1["ao_radius"], seed=99)
    assert 0.2 < ref.mean() < 0.95
    miss = orc.trace(*bvh.buffers_view(), prim)["prim"] < 0
    assert miss.any() and not miss.all()
    samples, errs, expect = [4, 16, 64], [], []
    for S in samples:
        ao = it.render_ao(cam, AmbientOcclusionIntegratorParams(samples=S, radius=C1["ao_radius"], seed=5)).cpu().numpy()
        g = ao[pix].astype(np.float64)
        assert (g[miss] == 0.0).all() and (ref[miss] == 0.0).all()  # primary misses contribute 0
        assert ((g >= 0.0) & (g <= 1.0)).all()
        errs.append(float(np.sqrt(np.mean((g - ref) ** 2)) / ref.mean()))
        # An unbiased S-sample estimate of an occlusion probability p has RMSE
        # sqrt(p (1 - p) / S): the measured error must be that and no more.
        expect.append(float(np.sqrt(np.mean(ref * (1.0 - ref)) / S) / ref.mean()))
    print("AO rel RMSE", dict(zip(samples, errs)), "binomial", dict(zip(samples, expect)))
    assert all(e <= 1.15 * x for e, x in zip(errs, expect))
    assert -0.65 <= _slope(samples, errs) <= -0.35


def _room(rb, n_spheres=60):
    return rb.RoomScene(seed=2, n_boxes=10, n_spheres=n_spheres, sphere_subdiv=2, n_lights=1, emission=10.0)


def test_pt_converges_to_host_reference(rb, orc, cuda):
    from renderbox2_b200.configs import CONFIG2 as C2
    from renderbox2_b200.render import DeviceScene, Integrator, PathIntegratorParams
    room = _room(rb)
    bvh = rb.BVH(room)
    it = Integrator(rb.CudaTracer(bvh), DeviceScene(room))
    W, H = 96, 54
    cam = rb.PerspectiveCamera(C2["eye"], C2["lookat"], C2["up"], (W, H), C2["fov"])
    step = 3
    ii, jj = np.meshgrid(np.arange(0, W, step), np.arange(0, H, step))
    pix = (jj * W + ii).ravel()
    ref_spp = 4096
    rng = np.random.Generator(np.random.PCG64(17))
    xy = (np.repeat(np.stack([ii.ravel(), jj.ravel()], 1), ref_spp, axis=0) +
          rng.uniform(0, 1, size=(pix.size * ref_spp, 2))).astype(np.float32)
    rays = orc.ref_camera_rays(C2["eye"], C2["lookat"], C2["up"], W, H, C2["fov"], xy)
    L = orc.pt(bvh.buffers_view(), room.vertices, room.indices, room.material_ids, room.albedo, room.emission,
               room.light_ids_to_primitive_ids, rays, C2["max_depth"], C2["rr_start"], C2["rr_prob"], seed=23)
    ref = L.reshape(pix.size, ref_spp, 3).mean(axis=1)
    assert ref.mean() > 0.0
    spps, errs = [16, 64, 256], []
    for spp in spps:
        img = it.render_pt(cam, PathIntegratorParams(spp=spp, max_depth=C2["max_depth"], rr_start=C2["rr_start"],
                                                      rr_prob=C2["rr_prob"], seed=31)).cpu().numpy()
        g = img[pix].astype(np.float64)
        assert np.isfinite(g).all() and (g >= 0).all()
        errs.append(float(np.sqrt(np.mean((g - ref) ** 2)) / ref.mean()))
    print("PT rel RMSE", dict(zip(spps, errs)), "stats", it.stats())
    assert errs[1] <= 0.25
    assert -0.65 <= _slope(spps, errs) <= -0.35


def test_pt_is_deterministic(rb, cuda):
    from renderbox2_b200.configs import CONFIG2 as C2
    from renderbox2_b200.render import DeviceScene, Integrator, PathIntegratorParams
    room = _room(rb, n_spheres=20)
    it = Integrator(rb.CudaTracer(rb.BVH(room)), DeviceScene(room))
    cam = rb.PerspectiveCamera(C2["eye"], C2["lookat"], C2["up"], (64, 36), C2["fov"])
    p = PathIntegratorParams(spp=8, seed=3, spp_per_wave=2)
    a = it.render_pt(cam, p).clone()
    b = it.render_pt(cam, p)
    assert cuda.equal(a, b)


def _bdpt_setup(rb, orc, W=96, H=54, step=3, n_iter=2048, n_light=2048):
    from renderbox2_b200.configs import CONFIG2 as C2
    room = _room(rb)
    bvh = rb.BVH(room)
    ii, jj = np.meshgrid(np.arange(0, W, step), np.arange(0, H, step))
    pix = (jj * W + ii).ravel()
    rng = np.random.Generator(np.random.PCG64(41))
    base = np.tile(np.stack([ii.ravel(), jj.ravel()], 1), (n_iter, 1))
    xy = (base + rng.uniform(0, 1, size=base.shape)).astype(np.float32)
    rays = orc.ref_camera_rays(C2["eye"], C2["lookat"], C2["up"], W, H, C2["fov"], xy)
    return room, bvh, pix, rays, C2


def test_bdpt_converges_to_host_reference(rb, orc, cuda):
    """Config 3 estimator (path length 6, one cached-vertex connection per
    camera vertex) against the FP64 host BDPT.  Bar: relative RMSE <= 0.8 at
    64 spp and slope -0.5 +- 0.15.  (Uniform 1/k strategy weights leave the
    1/d^2 of short connections unbalanced, so BDPT's per-pixel noise at equal
    spp is about 3x the path tracer's on this scene; unbiasedness is checked by
    the slope here and by test_bdpt_and_pt_agree_on_expectation.)"""
    from renderbox2_b200.render import BidirectionalPathIntegratorLvcParams, DeviceScene, Integrator
    W, H = 96, 54
    n_iter = 2048
    room, bvh, pix, rays, C2 = _bdpt_setup(rb, orc, W, H, n_iter=n_iter)
    ref = orc.bdpt(bvh.buffers_view(), room.vertices, room.indices, room.material_ids, room.albedo, room.emission,
                   room.light_ids_to_primitive_ids, rays, pix.size, n_iter, 2048, 6, 1, 3, 0.95, seed=43)
    it = Integrator(rb.CudaTracer(bvh), DeviceScene(room))
    cam = rb.PerspectiveCamera(C2["eye"], C2["lookat"], C2["up"], (W, H), C2["fov"])
    spps, errs = [16, 64, 256], []
    for spp in spps:
        img = it.render_bdpt(cam, BidirectionalPathIntegratorLvcParams(spp=spp, max_path_length=6, connections=1,
                                                                       seed=47)).cpu().numpy()
        g = img[pix].astype(np.float64)
        assert np.isfinite(g).all() and (g >= 0).all()
        errs.append(float(np.sqrt(np.mean((g - ref) ** 2)) / ref.mean()))
    st = it.stats()
    print("BDPT rel RMSE", dict(zip(spps, errs)), "stats", st)
    assert st["connection_rays"] > 0 and st["light_rays"] > 0 and st["lvc_vertices"] > 0
    assert errs[1] <= 0.8
    assert -0.65 <= _slope(spps, errs) <= -0.35


def test_bdpt_and_pt_agree_on_expectation(rb, cuda):
    """Both estimators are unbiased for paths of at most 6 segments (PT with
    max_depth 4 covers exactly those), so their converged images agree: the
    image means must match to 3 %."""
    from renderbox2_b200.configs import CONFIG2 as C2
    from renderbox2_b200.render import (BidirectionalPathIntegratorLvcParams, DeviceScene, Integrator,
                                        PathIntegratorParams)
    room = _room(rb)
    it = Integrator(rb.CudaTracer(rb.BVH(room)), DeviceScene(room))
    cam = rb.PerspectiveCamera(C2["eye"], C2["lookat"], C2["up"], (160, 90), C2["fov"])
    bd = it.render_bdpt(cam, BidirectionalPathIntegratorLvcParams(spp=512, max_path_length=6, connections=2)).cpu().numpy()
    pt = it.render_pt(cam, PathIntegratorParams(spp=512, max_depth=4)).cpu().numpy()
    rel = np.abs(bd.mean(0) - pt.mean(0)) / pt.mean(0)
    print("BDPT vs PT mean rel diff", rel)
    assert (rel < 0.03).all()


def test_integrators_on_compressed_wide_layout(rb, cuda):
    """With the tracer switched to the compressed 8-wide layout the
    integrators trace through it; hits equal the binary traversal's except for
    ties in t, so AO, PT and BDPT images are the binary-layout images (all but
    a negligible fraction of pixels bit-identical)."""
    from renderbox2_b200.configs import CONFIG2 as C2
    from renderbox2_b200.render import (AmbientOcclusionIntegratorParams, BidirectionalPathIntegratorLvcParams,
                                        DeviceScene, Integrator, PathIntegratorParams)
    room = _room(rb)
    tr = rb.CudaTracer(rb.BVH(room))
    it = Integrator(tr, DeviceScene(room))
    cam = rb.PerspectiveCamera(C2["eye"], C2["lookat"], C2["up"], (160, 90), C2["fov"])

    def images():
        ao = it.render_ao(cam, AmbientOcclusionIntegratorParams(samples=8, radius=0.5)).cpu().numpy()
        pt = it.render_pt(cam, PathIntegratorParams(spp=8, max_depth=6)).cpu().numpy()
        bd = it.render_bdpt(cam, BidirectionalPathIntegratorLvcParams(spp=4, max_path_length=6)).cpu().numpy()
        return ao, pt, bd

    ref = images()
    assert tr.status() == 0
    tr.set_node_order(rb.NODE_ORDER_CW8)
    got = images()
    assert tr.status() == 0
    for name, a, b in zip(("ao", "pt", "bdpt"), ref, got):
        assert np.isfinite(b).all()
        diff = (a != b).reshape(a.shape[0], -1).any(axis=1).mean()
        print(name, "differing pixels", diff)
        assert diff <= 1e-3, name
    tr.set_node_order(rb.NODE_ORDER_DFS)


@pytest.mark.parametrize("layered", [False, True])
def test_bdpt_waves_are_bit_identical(rb, cuda, layered):
    """BDPT runs several iterations per wave, each with its own light-vertex
    cache range; with the same random keys, the unfiltered image and the ray
    counts equal those of one iteration at a time, for any wave size."""
    from renderbox2_b200.configs import CONFIG2 as C2
    from renderbox2_b200.render import BidirectionalPathIntegratorLvcParams, DeviceScene, Integrator
    if layered:
        from test_gpu_material import _glossy_room
        room, mats = _glossy_room(rb)
        ds = DeviceScene(room, materials=mats)
    else:
        room = _room(rb)
        ds = DeviceScene(room)
    it = Integrator(rb.CudaTracer(rb.BVH(room)), ds)
    W, H = 160, 90
    cam = rb.PerspectiveCamera(C2["eye"], C2["lookat"], C2["up"], (W, H), C2["fov"])
    p = BidirectionalPathIntegratorLvcParams(spp=8, max_path_length=6, connections=2, num_light_paths=10_000, seed=5)
    imgs, stats = [], []
    for wave in (W * H, 3 * W * H, 0):   # 1 iteration per wave, 3 (3 + 3 + 2), all 8 (default budget)
        it.set_wave(wave)
        imgs.append(it.render_bdpt(cam, p).cpu())
        st = it.stats()
        stats.append({k: st[k] for k in ("primary_rays", "extension_rays", "shadow_rays", "connection_rays",
                                         "light_rays", "lvc_vertices")})
    assert imgs[0].float().mean() > 0
    for k in (1, 2):
        assert cuda.equal(imgs[0], imgs[k]), f"wave {k}"
        assert stats[0] == stats[k]


def test_far_camera_on_the_compressed_layout(rb, cuda):
    """The compressed 8-wide boxes' margin covers slab rounding for ray
    origins within 128 x the scene's largest coordinate; integrators trace
    camera rays from a camera beyond that through the binary buffer, so with
    the camera 1000 scene units away the AO and path-traced images equal the
    binary layout's (secondary rays start in the scene; ties aside)."""
    from renderbox2_b200.render import (AmbientOcclusionIntegratorParams, DeviceScene, Integrator,
                                        PathIntegratorParams)
    from renderbox2_b200.serve import lit_heightfield
    scene = lit_heightfield(21, 60_000)
    tr = rb.CudaTracer(rb.BVH(scene))
    it = Integrator(tr, DeviceScene(scene))
    # 1000 units away, a field of view that frames the unit field.  The camera
    # mirrors world x (the reference's scale(-1, 1, 1) in camera_to_world), so
    # eye and look-at x are negated to look at x = 0.5; at this 17.5-degree
    # elevation the field covers about a third of the frame (CPU oracle: 34 %).
    cam = rb.PerspectiveCamera((-0.5, 300.0, -950.0), (-0.5, 0.1, 0.5), (0, 1, 0), (96, 96), 0.06)

    def images():
        ao = it.render_ao(cam, AmbientOcclusionIntegratorParams(samples=8, radius=0.05)).cpu().numpy()
        pt = it.render_pt(cam, PathIntegratorParams(spp=4, max_depth=4)).cpu().numpy()
        return ao, pt

    ref = images()
    assert (ref[0] > 0).mean() > 0.25 and ref[1].mean() > 0.0   # the field is in the frame and lit
    tr.set_node_order(rb.NODE_ORDER_CW8)
    got = images()
    assert tr.status() == 0
    for name, a, b in zip(("ao", "pt"), ref, got):
        diff = (a != b).reshape(a.shape[0], -1).any(axis=1).mean()
        print(name, "differing pixels", diff)
        assert diff <= 2e-3, name
    tr.set_node_order(rb.NODE_ORDER_DFS)


def test_pt_progressive_resume_matches_one_render(rb, cuda):
    """Progressive path tracing: 20 + 20 + 24 samples added to running sums
    (with a host round trip of the sums between calls, as a checkpoint would
    do) give the same bits as one 64-sample render with the same seed; with a
    Gaussian film filter the same samples agree within float rounding."""
    import torch

    from renderbox2_b200.configs import CONFIG2 as C2
    from renderbox2_b200.render import DeviceScene, Filter, Integrator, PathIntegratorParams
    room = _room(rb, n_spheres=20)
    it = Integrator(rb.CudaTracer(rb.BVH(room)), DeviceScene(room))
    W, H = 64, 36
    cam = rb.PerspectiveCamera(C2["eye"], C2["lookat"], C2["up"], (W, H), C2["fov"])
    for filt in (None, Filter("gaussian", 2.0, 2.0, 2.0)):
        it.set_filter(filt)
        whole = it.render_pt(cam, PathIntegratorParams(spp=64, max_depth=5, seed=9, spp_per_wave=16)).clone()
        sums = torch.zeros((W * H * 4,), dtype=torch.float32, device="cuda")
        first = 0
        for spp in (20, 20, 24):
            img = it.render_pt_progressive(cam, PathIntegratorParams(spp=spp, max_depth=5, seed=9), first, sums)
            first += spp
            sums = sums.cpu().cuda()  # checkpoint: the state leaves the device and comes back
        torch.cuda.synchronize()
        if filt is None:
            assert cuda.equal(img, whole)
        else:
            assert torch.allclose(img, whole, rtol=1e-5, atol=1e-7)
    it.set_filter(None)
    with pytest.raises(rb.Rb2Error):
        it.render_pt_progressive(cam, PathIntegratorParams(spp=4), 0,
                                 torch.zeros((W * H * 4 + 1,), dtype=torch.float32, device="cuda")[1:])
