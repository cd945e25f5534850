"""Reference-compatibility modes on the GPU against the oracle's FP64
restatements of the same modes.

Each switch reproduces one behaviour of the reference that the integrators
otherwise correct: the AO direction formula (core/montecarlo.cu:133-151), the
path tracer's Russian-roulette divisor 1 - q (integrators/integrator_path.cu:
232-244) and its NEE re-seeding (:113), and the reference's own BDPT estimator
(integrators/integrator_bdpt_lvc_sk.cu:47-514: preparation pass sizing the
cache, 1 / ((bounce + 1) + depth) connection weights, full-weight NEE,
separate light and camera depths, DiffuseAreaLight::Le emission).

Bars, as for the default estimators (tests/test_gpu_render.py): the GPU image
converges to the FP64 host image of the same mode (relative RMSE below the
stated bound at 64 samples, log-log slope -0.5 +- 0.15, i.e. no bias), and the
mode's converged mean differs from the default mode's by more than the noise
(the switch really changes the estimator)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _slope(samples, errs):
    return float(np.polyfit(np.log(samples), np.log(errs), 1)[0])


def _room(rb):
    return rb.RoomScene(seed=2, n_boxes=10, n_spheres=60, sphere_subdiv=2, n_lights=1, emission=10.0)


def _grid(W, H, step):
    ii, jj = np.meshgrid(np.arange(0, W, step), np.arange(0, H, step))
    return ii, jj, (jj * W + ii).ravel()


def test_ao_direction_compat(rb, orc, cuda):
    from renderbox2_b200.configs import CONFIG1 as C1
    from renderbox2_b200.render import COMPAT_AO_DIRECTION, AmbientOcclusionIntegratorParams, DeviceScene, Integrator
    scene = rb.heightfield_scene(seed=C1["seed"], grid_n=C1["grid_n"], n_boxes=C1["n_boxes"])
    bvh = rb.BVH(scene)
    it = Integrator(rb.CudaTracer(bvh), DeviceScene(scene))
    cam = rb.PerspectiveCamera(C1["eye"], C1["lookat"], C1["up"], (C1["width"], C1["height"]), C1["fov"])
    ii, jj, pix = _grid(512, 512, 16)
    xy = np.stack([ii.ravel() + 0.5, jj.ravel() + 0.5], 1).astype(np.float32)
    prim = orc.ref_camera_rays(C1["eye"], C1["lookat"], C1["up"], 512, 512, C1["fov"], xy)
    ref = orc.ao(bvh.buffers_view(), scene.vertices, scene.indices, prim, 8192, C1["ao_radius"], seed=99, compat=1)
    ref0 = orc.ao(bvh.buffers_view(), scene.vertices, scene.indices, prim, 8192, C1["ao_radius"], seed=99)
    samples, errs, expect = [4, 16, 64], [], []
    for S in samples:
        p = AmbientOcclusionIntegratorParams(samples=S, radius=C1["ao_radius"], seed=5, compat=COMPAT_AO_DIRECTION)
        g = it.render_ao(cam, p).cpu().numpy()[pix].astype(np.float64)
        assert ((g >= 0.0) & (g <= 1.0)).all()
        errs.append(float(np.sqrt(np.mean((g - ref) ** 2)) / ref.mean()))
        expect.append(float(np.sqrt(np.mean(ref * (1.0 - ref)) / S) / ref.mean()))
    print("AO compat rel RMSE", dict(zip(samples, errs)), "binomial", dict(zip(samples, expect)),
          "means compat / default", ref.mean(), ref0.mean())
    assert all(e <= 1.15 * x for e, x in zip(errs, expect))
    assert -0.65 <= _slope(samples, errs) <= -0.35
    assert abs(ref.mean() - ref0.mean()) / ref0.mean() > 0.03


def test_pt_roulette_divisor_and_nee_reseed_compat(rb, orc, cuda):
    from renderbox2_b200.configs import CONFIG2 as C2
    from renderbox2_b200.render import (COMPAT_NEE_RESEED, COMPAT_RR_DIVISOR, DeviceScene, Integrator,
                                        PathIntegratorParams)
    room = _room(rb)
    bvh = rb.BVH(room)
    it = Integrator(rb.CudaTracer(bvh), DeviceScene(room))
    W, H = 96, 54
    cam = rb.PerspectiveCamera(C2["eye"], C2["lookat"], C2["up"], (W, H), C2["fov"])
    ii, jj, pix = _grid(W, H, 3)
    ref_spp = 4096
    rng = np.random.Generator(np.random.PCG64(17))
    xy = (np.repeat(np.stack([ii.ravel(), jj.ravel()], 1), ref_spp, axis=0) +
          rng.uniform(0, 1, size=(pix.size * ref_spp, 2))).astype(np.float32)
    rays = orc.ref_camera_rays(C2["eye"], C2["lookat"], C2["up"], W, H, C2["fov"], xy)
    compat = COMPAT_RR_DIVISOR | COMPAT_NEE_RESEED
    L = orc.pt(bvh.buffers_view(), room.vertices, room.indices, room.material_ids, room.albedo, room.emission,
               room.light_ids_to_primitive_ids, rays, C2["max_depth"], C2["rr_start"], C2["rr_prob"], seed=23,
               compat=compat)
    ref = L.reshape(pix.size, ref_spp, 3).mean(axis=1)
    spps, errs = [16, 64, 256], []
    for spp in spps:
        p = PathIntegratorParams(spp=spp, max_depth=C2["max_depth"], rr_start=C2["rr_start"], rr_prob=C2["rr_prob"],
                                 seed=31, compat=compat)
        g = it.render_pt(cam, p).cpu().numpy()[pix].astype(np.float64)
        assert np.isfinite(g).all() and (g >= 0).all()
        errs.append(float(np.sqrt(np.mean((g - ref) ** 2)) / ref.mean()))
    full = PathIntegratorParams(spp=1024, max_depth=C2["max_depth"], rr_start=C2["rr_start"], rr_prob=C2["rr_prob"],
                                seed=37)
    m_default = it.render_pt(cam, full).cpu().numpy().mean()
    full.compat = compat
    m_compat = it.render_pt(cam, full).cpu().numpy().mean()
    print("PT compat rel RMSE", dict(zip(spps, errs)), "means compat / default", m_compat, m_default)
    assert errs[1] <= 0.3
    assert -0.65 <= _slope(spps, errs) <= -0.35
    assert (m_default - m_compat) / m_default > 0.01   # dividing by 1 - q loses energy here


def _bdpt_reference_params(spp, seed, **kw):
    from renderbox2_b200.render import BidirectionalPathIntegratorLvcParams
    # The reference's integrator file (integrators/integrator_bdpt_lvc.xml), with
    # config 3's one connection per camera vertex and 2048 light paths.
    p = dict(spp=spp, seed=seed, estimator="reference", num_prep_paths=10000, num_light_paths=2048,
             num_light_path_max_depth=8, light_path_rrstart=4, num_cam_path_max_depth=8, cam_path_rrstart=4,
             cam_path_rrprob=0.3, num_cam_path_sample_connections=10, connections=1, mode="sk")
    p.update(kw)
    return BidirectionalPathIntegratorLvcParams(**p)


def test_bdpt_reference_estimator_converges_to_host(rb, orc, cuda):
    """In a room 5 units on a side, where the light's triangles have area 0.5,
    the reference's triangle-area quirk (every area 0.5) is neutral and the
    estimator's variance is moderate.  (In the unit room its light-sample pdf
    is 25x too small and its light subpaths carry 25x their power, so its
    connections are heavy-tailed: two 2048-iteration host images differ by
    7 % RMSE there, against 1.4 % here.)"""
    from renderbox2_b200.configs import CONFIG2 as C2
    from renderbox2_b200.render import BidirectionalPathIntegratorLvcParams, DeviceScene, Integrator
    rs = 5.0
    room = rb.RoomScene(seed=2, n_boxes=10, n_spheres=60, sphere_subdiv=2, n_lights=1, emission=10.0, room_size=rs)
    bvh = rb.BVH(room)
    eye, look = [x * rs for x in C2["eye"]], [x * rs for x in C2["lookat"]]
    W, H = 96, 54
    ii, jj, pix = _grid(W, H, 3)
    n_iter = 2048
    rng = np.random.Generator(np.random.PCG64(41))
    base = np.tile(np.stack([ii.ravel(), jj.ravel()], 1), (n_iter, 1))
    xy = (base + rng.uniform(0, 1, size=base.shape)).astype(np.float32)
    rays = orc.ref_camera_rays(eye, look, C2["up"], W, H, C2["fov"], xy)
    ref = orc.bdpt_ref(bvh.buffers_view(), room.vertices, room.indices, room.material_ids, room.albedo,
                       room.emission, room.light_ids_to_primitive_ids, rays, pix.size, n_iter, 10000, 2048, 8, 8, 4,
                       0.3, 1, seed=43)
    it = Integrator(rb.CudaTracer(bvh), DeviceScene(room))
    cam = rb.PerspectiveCamera(eye, look, C2["up"], (W, H), C2["fov"])
    spps, errs = [16, 64, 256], []
    for spp in spps:
        g = it.render_bdpt(cam, _bdpt_reference_params(spp, 47)).cpu().numpy()[pix].astype(np.float64)
        assert np.isfinite(g).all() and (g >= 0).all()
        errs.append(float(np.sqrt(np.mean((g - ref) ** 2)) / ref.mean()))
    st = it.stats()
    print("BDPT reference-estimator rel RMSE", dict(zip(spps, errs)), "stats", st)
    assert st["connection_rays"] > 0 and st["light_rays"] > 0 and st["lvc_vertices"] > 0
    assert errs[1] <= 0.8
    assert -0.65 <= _slope(spps, errs) <= -0.35
    # The reference's estimator is not the unbiased one: in the unit room, where
    # the lights' triangles have area 0.02, its 0.5-area quirk makes the
    # converged image many times brighter.
    room1 = _room(rb)
    it1 = Integrator(rb.CudaTracer(rb.BVH(room1)), DeviceScene(room1))
    cam1 = rb.PerspectiveCamera(C2["eye"], C2["lookat"], C2["up"], (W, H), C2["fov"])
    ref_mean = it1.render_bdpt(cam1, _bdpt_reference_params(256, 53)).cpu().numpy().mean()
    unb_mean = it1.render_bdpt(cam1, BidirectionalPathIntegratorLvcParams(spp=256, max_path_length=9, connections=1,
                                                                          num_light_paths=2048, seed=53)).cpu().numpy().mean()
    print("BDPT unit-room means reference / unbiased", ref_mean, unb_mean)
    assert ref_mean > 5.0 * unb_mean


def test_bdpt_reference_params_struct(rb, cuda):
    """Every field of the reference's BidirectionalPathIntegratorLvcParams is
    accepted; the three kernel organisations (sk, mk, sort) run one
    estimator (identical images); sample_M, which no reference kernel reads,
    does not change the image; fields out of range are rejected."""
    from renderbox2_b200.configs import CONFIG2 as C2
    from renderbox2_b200.render import DeviceScene, Integrator
    room = _room(rb)
    it = Integrator(rb.CudaTracer(rb.BVH(room)), DeviceScene(room))
    cam = rb.PerspectiveCamera(C2["eye"], C2["lookat"], C2["up"], (64, 36), C2["fov"])
    imgs = [it.render_bdpt(cam, _bdpt_reference_params(4, 3, mode=m)).cpu() for m in ("sk", "mk", "sort")]
    imgs.append(it.render_bdpt(cam, _bdpt_reference_params(4, 3, num_cam_path_sample_connections=1)).cpu())
    assert float(imgs[0].mean()) > 0.0
    for k in range(1, len(imgs)):
        assert cuda.equal(imgs[0], imgs[k])
    # no preparation pass: the cache is never capped
    assert float(it.render_bdpt(cam, _bdpt_reference_params(4, 3, num_prep_paths=0)).cpu().mean()) > 0.0
    for bad in (dict(cam_path_rrprob=1.0), dict(num_light_path_max_depth=0), dict(connections=9)):
        with pytest.raises(rb.Rb2Error) as e:
            it.render_bdpt(cam, _bdpt_reference_params(4, 3, **bad))
        assert e.value.code == 1
