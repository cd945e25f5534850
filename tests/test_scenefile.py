"""Scene-file loading (the reference's XML schema and OBJ): CPU tests of the
parse semantics, material numbering and errors."""
from pathlib import Path

import numpy as np
import pytest

DATA = Path(__file__).resolve().parent / "data"


def test_obj_objects_faces_and_indices(rb):
    sf = rb.load_scene_file(str(DATA / "box_scene.obj"))
    s = sf.scene
    names = [m[0] for m in sf.meshes]
    assert names == ["floor", "ceiling", "back", "left", "right", "front", "block", "lamp"]
    counts = {m[0]: m[2] for m in sf.meshes}
    # quads are fan-triangulated; v, v/vt, v/vt/vn, v//vn and negative indices parse
    assert counts == {"floor": 2, "ceiling": 2, "back": 2, "left": 2, "right": 2, "front": 2, "block": 10, "lamp": 2}
    assert s.vertices.shape == (36, 3) and s.indices.shape == (24, 3)
    assert s.indices.max() == 35
    assert list(s.indices[0]) == [0, 3, 2] and list(s.indices[1]) == [0, 2, 1]   # fan from the first vertex
    left = sf.meshes[3]
    assert list(s.indices[left[1]]) == [12, 13, 14]                              # -4 -3 -2 relative indices
    assert (s.material_ids == 0).all() and sf.bsdf_types == ["lambertian"] and sf.camera is None
    assert s.num_lights == 0


def test_xml_materials_lights_camera(rb):
    sf = rb.load_scene_file(str(DATA / "box_scene.xml"))
    s = sf.scene
    assert sf.bsdf_types == ["lambertian", "lambertian", "orennayar", "emitter"]
    np.testing.assert_array_equal(s.albedo, np.array([[0.8, 0.8, 0.8], [0.75, 0.1, 0.1], [0.1, 0.7, 0.1], [0, 0, 0]],
                                                     np.float32))
    np.testing.assert_array_equal(s.emission[3], np.float32([12, 12, 12]))
    mat_of = {name: set(s.material_ids[first:first + n].tolist()) for name, first, n in sf.meshes}
    assert mat_of["left"] == {1} and mat_of["right"] == {2} and mat_of["lamp"] == {3}
    assert mat_of["front"] == {0}          # not named by the file: material 0
    assert s.num_lights == 2 and set(s.light_ids_to_primitive_ids.tolist()) == {22, 23}
    assert sf.camera == {"eye": [-0.5, 0.5, np.float32(0.02)], "lookat": [-0.5, 0.5, 0.5], "up": [0.0, 1.0, 0.0],
                         "fov": 70.0}
    # the loaded scene builds
    bvh = rb.BVH(s)
    assert bvh.counts().n_tris == 24


@pytest.mark.parametrize("text,needle", [
    ("<scene><files><count>1</count></files></scene>", "file"),
    ("<scene><files><file>missing.obj</file></files></scene>", "cannot open"),
    ("<scene><files><file>box_scene.obj</file></files>", "missing </scene>"),
    ("<scene><files><file>box_scene.obj</file></files><material><name>m</name><bsdf><bxdf><type>velvet</type>"
     "</bxdf></bsdf></material></scene>", "unknown bxdf"),
    ("<scene><files><file>box_scene.obj</file></files><object><name>floor</name><material>nope</material></object>"
     "</scene>", "unknown material"),
    ("<root/>", "not <scene>"),
    ("<scene><a>&bogus;</a></scene>", "entity"),
])
def test_xml_errors(rb, tmp_path, text, needle):
    import shutil
    shutil.copy(DATA / "box_scene.obj", tmp_path / "box_scene.obj")
    p = tmp_path / "s.xml"
    p.write_text(text)
    with pytest.raises(rb.Rb2Error, match=needle):
        rb.load_scene_file(str(p))


@pytest.mark.parametrize("text,needle", [
    ("v 0 0 0\nv 1 0 0\nf 1 2\n", "fewer than three"),
    ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4\n", "out of range"),
    ("v 0 0\n", "three coordinates"),
    ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 x\n", "bad face vertex"),
    ("# nothing\n", "no faces"),
])
def test_obj_errors(rb, tmp_path, text, needle):
    p = tmp_path / "m.obj"
    p.write_text(text)
    with pytest.raises(rb.Rb2Error, match=needle):
        rb.load_scene_file(str(p))


def test_obj_geometry_before_first_object(rb, tmp_path):
    p = tmp_path / "m.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\no tri2\nv 0 0 1\nf 1 2 4\n")
    sf = rb.load_scene_file(str(p))
    assert [m[0] for m in sf.meshes] == ["default", "tri2"] and sf.scene.indices.shape == (2, 3)
