"""Seeded synthetic scenes, ray sets and the perspective camera (librb2)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._native import Camera as _Camera
from ._native import check, lib
from .accel import Scene, _ptr, _stream_handle


def heightfield_scene(seed: int = 1, grid_n: int = 256, amplitude: float = 0.2, n_boxes: int = 64,
                      box_min: float = 0.02, box_max: float = 0.1) -> Scene:
    """Value-noise heightfield over the unit square plus axis-aligned boxes."""
    L = lib()
    nv, nt = C.c_uint32(), C.c_uint32()
    check(L.rb2_gen_heightfield_counts(grid_n, n_boxes, C.byref(nv), C.byref(nt)))
    v = np.empty((nv.value, 3), np.float32)
    i = np.empty((nt.value, 3), np.uint32)
    check(L.rb2_gen_heightfield(seed, grid_n, amplitude, n_boxes, box_min, box_max, _ptr(v), _ptr(i)))
    s = Scene()
    s.vertices, s.indices = v, i
    s.material_ids = np.zeros((nt.value,), np.uint32)
    return s


def heightfield_for_triangles(seed: int, n_tris: int, n_boxes: int = 64) -> Scene:
    """Heightfield whose grid is sized to about n_tris triangles (grid n =
    round(sqrt((T - 12*boxes) / 2)))."""
    n = max(1, int(round(np.sqrt(max(2, n_tris - 12 * n_boxes) / 2.0))))
    return heightfield_scene(seed=seed, grid_n=n, n_boxes=n_boxes)


class RoomScene(Scene):
    """Closed room with boxes, icospheres and quad area lights.

    material_ids index `albedo` / `emission`; lights are the emitter
    triangles (two per quad)."""

    def __init__(self, seed=1, n_boxes=100, n_spheres=2000, sphere_subdiv=2, rmin=0.01, rmax=0.2, n_lights=1,
                 emission=10.0, room_size=1.0):
        """room_size scales the whole room (walls, boxes, lights); sphere
        radii rmin..rmax are absolute, so a 10-unit room holds 2000 spheres
        of radius up to 0.2 with space between them."""
        super().__init__()
        L = lib()
        nv, nt = C.c_uint32(), C.c_uint32()
        check(L.rb2_gen_room_counts(n_boxes, n_spheres, sphere_subdiv, n_lights, C.byref(nv), C.byref(nt)))
        v = np.empty((nv.value, 3), np.float32)
        i = np.empty((nt.value, 3), np.uint32)
        m = np.empty((nt.value,), np.uint32)
        check(L.rb2_gen_room(seed, n_boxes, n_spheres, sphere_subdiv, rmin / room_size, rmax / room_size, n_lights,
                             _ptr(v), _ptr(i), _ptr(m)))
        if room_size != 1.0:
            v *= np.float32(room_size)
        self.vertices, self.indices, self.material_ids = v, i, m
        n_mat = 6 + n_boxes + n_spheres + n_lights
        rng = np.random.Generator(np.random.PCG64(seed))
        self.albedo = rng.uniform(0.2, 0.8, size=(n_mat, 3)).astype(np.float32)
        self.emission = np.zeros((n_mat, 3), np.float32)
        first_light_mat = n_mat - n_lights
        self.albedo[first_light_mat:] = 0.0
        self.emission[first_light_mat:] = emission
        self.light_ids_to_primitive_ids = np.nonzero(m >= first_light_mat)[0].astype(np.uint32)


def surface_rays(scene: Scene, seed: int, n: int, offset_scale: float = 1e-4, anyhit_fraction: float = 0.5):
    """Incoherent diffuse-bounce rays from the scene's surfaces.  Returns
    (rays (n, 8) float32, flags (n,) uint8 with 1 = any-hit)."""
    rays = np.empty((n, 8), np.float32)
    flags = np.empty((n,), np.uint8)
    v = np.ascontiguousarray(scene.vertices, np.float32)
    i = np.ascontiguousarray(scene.indices, np.uint32)
    check(lib().rb2_gen_surface_rays(_ptr(v), v.shape[0], _ptr(i), i.shape[0], seed, n, offset_scale,
                                     anyhit_fraction, _ptr(rays), _ptr(flags)))
    return rays, flags


def pcg32(seed: int, stream: int, n: int) -> np.ndarray:
    out = np.empty((n,), np.uint32)
    check(lib().rb2_pcg32_fill(seed, stream, n, _ptr(out)))
    return out


class PerspectiveCamera:
    """PerspectiveCamera(position, lookat, up, resolution, horizontal_fov)
    (core/camera.h:40-95)."""

    def __init__(self, position, lookat, up, resolution, fov_deg):
        self.c = _Camera()
        e = np.asarray(position, np.float32)
        l_ = np.asarray(lookat, np.float32)
        u = np.asarray(up, np.float32)
        self.width, self.height = int(resolution[0]), int(resolution[1])
        check(lib().rb2_camera_init(C.byref(self.c), _ptr(e), _ptr(l_), _ptr(u), self.width, self.height,
                                    float(fov_deg)))

    def generate_rays(self, spp: int = 1, seed: int = 0, jitter: bool = False, out=None, stream=None):
        import torch
        n = self.width * self.height * spp
        if out is None:
            out = torch.empty((n, 8), dtype=torch.float32, device="cuda")
        check(lib().rb2_camera_rays(C.byref(self.c), spp, seed, 1 if jitter else 0, _ptr(out), _stream_handle(stream)))
        return out

    def generate_rays_at(self, raster_xy, out=None, stream=None):
        import torch
        n = raster_xy.shape[0]
        if out is None:
            out = torch.empty((n, 8), dtype=torch.float32, device=raster_xy.device)
        check(lib().rb2_camera_rays_at(C.byref(self.c), _ptr(raster_xy), n, _ptr(out), _stream_handle(stream)))
        return out
