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
    # the red wall (material 1) and the green wall (material 2) tint opposite halves
    a, b = img[:, : W // 2 - 8], img[:, W // 2 + 8:]
    da = a[..., 0].mean() - a[..., 1].mean()
    db = b[..., 0].mean() - b[..., 1].mean()
    assert da * db < 0 and min(abs(da), abs(db)) > 0.005
    st = it.stats()
    assert st["shadow_rays"] > 0 and st["extension_rays"] > 0
