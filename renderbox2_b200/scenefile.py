"""Scene files: the reference's XML scene description and Wavefront OBJ
(io/customfilereader.cpp:47-291, io/objfilereader.cpp:117-216), parsed by
librb2 (rb2_scene_file_load)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._native import MaterialDesc, check, lib
from .accel import Scene

BSDF_NAMES = {0: "lambertian", 1: "orennayar", 2: "mirror", 3: "glass", 4: "microfacet", 5: "emitter"}


class SceneFileInfo(C.Structure):
    _fields_ = [("n_vertices", C.c_uint32), ("n_triangles", C.c_uint32), ("n_materials", C.c_uint32),
                ("n_lights", C.c_uint32), ("n_meshes", C.c_uint32), ("has_camera", C.c_int32),
                ("eye", C.c_float * 3), ("lookat", C.c_float * 3), ("up", C.c_float * 3), ("fov_deg", C.c_float)]


def _sigs(L):
    P = C.c_void_p
    if getattr(L, "_rb2_scenefile_sigs", False):
        return
    L.rb2_scene_file_load.argtypes, L.rb2_scene_file_load.restype = [C.c_char_p, C.POINTER(P)], C.c_int
    L.rb2_scene_file_info_get.argtypes, L.rb2_scene_file_info_get.restype = [P, C.POINTER(SceneFileInfo)], C.c_int
    for name, t in (("vertices", C.c_float), ("indices", C.c_uint32), ("tri_material", C.c_uint32),
                    ("albedo", C.c_float), ("emission", C.c_float), ("bsdf_types", C.c_uint32)):
        fn = getattr(L, "rb2_scene_file_" + name)
        fn.argtypes, fn.restype = [P], C.POINTER(t)
    L.rb2_scene_file_mesh.argtypes = [P, C.c_uint32, C.POINTER(C.c_char_p), C.POINTER(C.c_uint32),
                                      C.POINTER(C.c_uint32)]
    L.rb2_scene_file_mesh.restype = C.c_int
    L.rb2_scene_file_free.argtypes, L.rb2_scene_file_free.restype = [P], None
    L.rb2_scene_file_materials.argtypes, L.rb2_scene_file_materials.restype = [P], C.POINTER(MaterialDesc)
    L._rb2_scenefile_sigs = True


class SceneFile:
    """A loaded scene file: `scene` (Scene with material ids, per-material
    albedo / emission, the layered material descriptions `materials` and the
    emissive-triangle list), `camera` (dict or None), `bsdf_types` (first
    layer's bxdf per material) and `meshes` (name, first triangle, count)."""

    def __init__(self, path: str):
        L = lib()
        _sigs(L)
        h = C.c_void_p()
        check(L.rb2_scene_file_load(str(path).encode(), C.byref(h)))
        try:
            info = SceneFileInfo()
            check(L.rb2_scene_file_info_get(h, C.byref(info)))
            nv, nt, nm = info.n_vertices, info.n_triangles, info.n_materials

            def arr(fn, n, dt):
                return np.ctypeslib.as_array(fn(h), shape=(n,)).astype(dt, copy=True)

            s = Scene()
            s.vertices = arr(L.rb2_scene_file_vertices, 3 * nv, np.float32).reshape(-1, 3)
            s.indices = arr(L.rb2_scene_file_indices, 3 * nt, np.uint32).reshape(-1, 3)
            s.material_ids = arr(L.rb2_scene_file_tri_material, nt, np.uint32)
            s.albedo = arr(L.rb2_scene_file_albedo, 3 * nm, np.float32).reshape(-1, 3)
            s.emission = arr(L.rb2_scene_file_emission, 3 * nm, np.float32).reshape(-1, 3)
            types = arr(L.rb2_scene_file_bsdf_types, nm, np.uint32)
            mp = L.rb2_scene_file_materials(h)
            s.materials = (MaterialDesc * nm)(*[mp[i] for i in range(nm)])
            s.light_ids_to_primitive_ids = np.nonzero(types[s.material_ids] == 5)[0].astype(np.uint32)
            self.scene = s
            self.bsdf_types = [BSDF_NAMES[int(t)] for t in types]
            self.meshes = []
            for i in range(info.n_meshes):
                name, first, count = C.c_char_p(), C.c_uint32(), C.c_uint32()
                check(L.rb2_scene_file_mesh(h, i, C.byref(name), C.byref(first), C.byref(count)))
                self.meshes.append((name.value.decode(), first.value, count.value))
            self.camera = None
            if info.has_camera:
                self.camera = {"eye": list(info.eye), "lookat": list(info.lookat), "up": list(info.up),
                               "fov": float(info.fov_deg)}
        finally:
            L.rb2_scene_file_free(h)


def load_scene_file(path: str) -> SceneFile:
    return SceneFile(path)
