"""GPU parity of the film (filtered reconstruction) through the C ABI.

Bar: rb2_film_develop bit-identical to the oracle's restatement of the
reference's splat (oracle.film) for every filter; the path tracer with a
filter is deterministic, keeps the image mean, and with a box of half-width
0.5 equals the unfiltered image to float rounding."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _samples(W, H, spp, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    pix = np.arange(W * H)
    base = np.stack([pix % W, pix // W], 1).astype(np.float32)
    xy = (np.tile(base, (spp, 1)) + rng.uniform(0, 1, (spp * W * H, 2))).astype(np.float32)
    xy = np.minimum(xy, np.nextafter(np.tile(base, (spp, 1)) + 1, 0, dtype=np.float32))
    L = rng.exponential(1.0, (spp * W * H, 4)).astype(np.float32)
    return xy, L


@pytest.mark.parametrize("kind,xw,yw,alpha", [("none", 0.5, 0.5, 0.0), ("box", 0.5, 0.5, 0.0), ("box", 1.0, 1.5, 0.0),
                                              ("triangle", 2.0, 2.0, 0.0), ("gaussian", 2.0, 2.0, 2.0),
                                              ("gaussian", 1.3, 3.1, 0.7)])
def test_film_develop_equals_oracle(rb, orc, cuda, kind, xw, yw, alpha):
    from renderbox2_b200.render import Filter, film_develop
    torch = cuda
    W, H, spp = 37, 23, 5
    xy, L = _samples(W, H, spp, seed=7)
    # Edge positions: exact pixel corners and the last float below the next pixel.
    xy[0] = (0.0, 0.0)
    xy[1] = (1.0, 0.0)
    got = film_develop(Filter(kind, xw, yw, alpha), W, H, spp, torch.from_numpy(xy).cuda(),
                       torch.from_numpy(L).cuda()).cpu().numpy()
    want = orc.film(kind, xw, yw, alpha, W, H, spp, xy, L)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def _pt_setup(rb):
    from renderbox2_b200.configs import CONFIG2 as C2
    from renderbox2_b200.render import DeviceScene, Integrator
    room = rb.RoomScene(seed=2, n_boxes=10, n_spheres=40, sphere_subdiv=2, n_lights=1, emission=10.0)
    it = Integrator(rb.CudaTracer(rb.BVH(room)), DeviceScene(room))
    cam = rb.PerspectiveCamera(C2["eye"], C2["lookat"], C2["up"], (160, 90), C2["fov"])
    return it, cam


def test_filtered_path_tracing(rb, cuda):
    from renderbox2_b200.render import Filter, PathIntegratorParams
    torch = cuda
    it, cam = _pt_setup(rb)
    p = PathIntegratorParams(spp=16, max_depth=5, seed=3)
    plain = it.render_pt(cam, p).cpu().numpy()
    it.set_filter(Filter("box", 0.5, 0.5))
    box = it.render_pt(cam, p).cpu().numpy()
    # Equal except where a sample's raster position rounded onto a pixel edge:
    # the box of half-width 0.5 then also reaches the neighbour (as the
    # reference's window test does), about one sample in 2^17 here.
    close = np.isclose(box, plain, rtol=2e-5, atol=1e-6).all(axis=1)
    assert (~close).sum() <= 8, (~close).sum()
    it.set_filter(Filter("gaussian", 2.0, 2.0, 2.0))
    g1 = it.render_pt(cam, p).cpu().numpy()
    g2 = it.render_pt(cam, p).cpu().numpy()
    assert np.array_equal(g1, g2)                                      # deterministic
    assert abs(g1.mean() / plain.mean() - 1.0) < 0.02                  # energy kept
    # smoother: less pixel-to-pixel variation than the unfiltered image
    img_p, img_g = plain.reshape(90, 160, 3), g1.reshape(90, 160, 3)
    assert np.abs(np.diff(img_g, axis=1)).mean() < 0.7 * np.abs(np.diff(img_p, axis=1)).mean()
    # several waves (spp_per_wave) give the same filtered image
    g3 = it.render_pt(cam, PathIntegratorParams(spp=16, max_depth=5, seed=3, spp_per_wave=4)).cpu().numpy()
    assert np.allclose(g3, g1, rtol=1e-5, atol=1e-6)
    it.set_filter(None)
    again = it.render_pt(cam, p).cpu().numpy()
    assert np.array_equal(again, plain)
    del torch


def test_filtered_bdpt_keeps_mean(rb, cuda):
    from renderbox2_b200.render import BidirectionalPathIntegratorLvcParams, Filter
    it, cam = _pt_setup(rb)
    p = BidirectionalPathIntegratorLvcParams(spp=8, max_path_length=5, connections=1, seed=5)
    plain = it.render_bdpt(cam, p).cpu().numpy()
    it.set_filter(Filter("triangle", 1.5, 1.5))
    tri = it.render_bdpt(cam, p).cpu().numpy()
    assert abs(tri.mean() / plain.mean() - 1.0) < 0.03
    assert np.isfinite(tri).all() and (tri >= 0).all()
