"""A scene loaded from the reference's XML schema renders on the B200: the
wavefront path tracer sees its materials and its light."""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
DATA = Path(__file__).resolve().parent / "data"


def test_render_loaded_xml_scene(rb, cuda):
    from renderbox2_b200.render import DeviceScene, Filter, Integrator, PathIntegratorParams
    sf = rb.load_scene_file(str(DATA / "box_scene.xml"))
    it = Integrator(rb.CudaTracer(rb.BVH(sf.scene)), DeviceScene(sf.scene))
    c = sf.camera
    W, H = 96, 96
    cam = rb.PerspectiveCamera(c["eye"], c["lookat"], c["up"], (W, H), c["fov"])
    it.set_filter(Filter("gaussian", 1.5, 1.5, 2.0))
    img = it.render_pt(cam, PathIntegratorParams(spp=64, max_depth=6, seed=9)).cpu().numpy().reshape(H, W, 3)
    assert np.isfinite(img).all() and img.mean() > 0.02
    # the red wall (material 1) and the green wall (material 2) tint the image's halves
    # (the reference camera mirrors x: the left wall appears on the image's right)
    right, left = img[:, W // 2 + 8:], img[:, : W // 2 - 8]
    assert right[..., 0].mean() > right[..., 1].mean() and left[..., 1].mean() > left[..., 0].mean()
    st = it.stats()
    assert st["shadow_rays"] > 0 and st["extension_rays"] > 0
