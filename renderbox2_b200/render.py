"""Device scene and wavefront integrators (AO, path tracing, BDPT).

Mirrors the reference's Integrator::render(Scene*, CudaTracer*, ...)
(core/integrator.h:44-66) with the parameter structs of core/params.h:88-131.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._native import AoParams, BdptLvcParams, DevScene, IsectBuffer, PtParams, RayCastParams, RenderStats, check, lib
from ._native import BsdfLayer as _BsdfLayer
from ._native import Filter as _Filter
from ._native import MaterialDesc as _MaterialDesc
from .accel import CudaTracer, Scene, _ptr, _stream_handle


BSDF_KINDS = {"lambertian": 0, "orennayar": 1, "mirror": 2, "glass": 3, "microfacet": 4}
FRESNEL_KINDS = {"dielectric": 0, "conductor": 1, "noop": 2}


@dataclass
class BsdfLayer:
    """One bxdf of a material (core/params.h:195-245)."""
    type: str = "lambertian"
    color: tuple = (0.5, 0.5, 0.5)
    sigma_deg: float = 0.0                 # Oren-Nayar
    etai: float = 1.0
    etat: float = 1.5                      # glass / dielectric Fresnel
    exponent: float = 20.0                 # Blinn microfacet
    fresnel: str = "noop"
    eta: tuple = (0.2, 0.9, 1.1)
    k: tuple = (3.9, 2.4, 2.2)             # conductor Fresnel

    def c_struct(self) -> _BsdfLayer:
        return _BsdfLayer(BSDF_KINDS[self.type], FRESNEL_KINDS[self.fresnel], (C.c_float * 3)(*self.color),
                          self.sigma_deg, self.etai, self.etat, self.exponent, (C.c_float * 3)(*self.eta),
                          (C.c_float * 3)(*self.k))


def material_descs(materials) -> "C.Array":
    """A ctypes array of rb2_material_desc from lists of BsdfLayer (an
    empty list = an emitter's material)."""
    arr = (_MaterialDesc * max(1, len(materials)))()
    for i, layers in enumerate(materials):
        assert len(layers) <= 4, "at most 4 layers"
        arr[i].n_layers = len(layers)
        for j, l in enumerate(layers):
            arr[i].layer[j] = l.c_struct()
    return arr


class DeviceScene:
    """Scene::gpu_prepare equivalent: vertices, triangles, materials, lights.
    `materials` (or the scene's own `materials` attribute): one list of
    BsdfLayer, or a ctypes rb2_material_desc array, per material."""

    def __init__(self, scene: Scene, albedo=None, emission=None, materials=None):
        v = np.ascontiguousarray(scene.vertices, np.float32)
        i = np.ascontiguousarray(scene.indices, np.uint32)
        m = np.ascontiguousarray(scene.material_ids, np.uint32)
        albedo = getattr(scene, "albedo", None) if albedo is None else albedo
        emission = getattr(scene, "emission", None) if emission is None else emission
        n_mat = int(max(m.max() + 1 if m.size else 1, 0 if albedo is None else len(albedo),
                        0 if emission is None else len(emission)))
        a = None if albedo is None else np.ascontiguousarray(albedo, np.float32).reshape(-1, 3)
        e = None if emission is None else np.ascontiguousarray(emission, np.float32).reshape(-1, 3)
        self._keep = (v, i, m, a, e)
        self._s = C.c_void_p()
        check(lib().rb2_scene_create(_ptr(v), v.shape[0], _ptr(i), i.shape[0], _ptr(m), n_mat, _ptr(a), _ptr(e),
                                     C.byref(self._s)))
        self.n_materials = n_mat
        materials = getattr(scene, "materials", None) if materials is None else materials
        if materials is not None:
            self.set_materials(materials)

    def set_materials(self, materials):
        arr = materials if isinstance(materials, C.Array) else material_descs(materials)
        check(lib().rb2_scene_set_materials(self._s, arr, len(arr)))

    def material_query(self, mat_ids, q, sample: bool = False, stream=None):
        """Device material evaluation (rb2_material_query): q (n, 9) float32
        device tensor; returns (n, 4) f/pdf or (n, 8) wi/f/pdf/specular."""
        import torch
        n = int(q.shape[0])
        out = torch.empty((n, 8 if sample else 4), dtype=torch.float32, device=q.device)
        check(lib().rb2_material_query(self._s, 1 if sample else 0, _ptr(mat_ids), _ptr(q), n, _ptr(out),
                                       _stream_handle(stream)))
        return out

    def __del__(self):
        s = getattr(self, "_s", None)
        if s and s.value and lib is not None:  # lib is None at interpreter shutdown
            lib().rb2_scene_destroy(s)
            self._s = C.c_void_p()

    @property
    def handle(self):
        return self._s

    def dev_view(self) -> dict:
        d = DevScene()
        check(lib().rb2_scene_dev_view(self._s, C.byref(d)))
        return {k: getattr(d, k) for k, _ in DevScene._fields_}


class IntersectionBuffer:
    """The reference's SoA IntersectionBuffer (core/intersection.h:63-80) as
    device tensors: position / geometric_normal / shading_normal /
    incoming_direction (3, n) float32, uv (n, 2) float32, primitive_id and
    primitive_material_id (n,) int32 (uint32 bits), front and intersected
    (n,) uint8, epsilon (n,) float32.  `fields` limits which are allocated
    (the others are skipped by the kernel)."""

    VEC = ("position", "geometric_normal", "shading_normal", "incoming_direction")
    ALL = VEC + ("uv", "primitive_id", "primitive_material_id", "front", "intersected", "epsilon")

    def __init__(self, n: int, device="cuda", fields=None):
        import torch
        self.n = n
        fields = self.ALL if fields is None else tuple(fields)
        self.t = {}
        for k in fields:
            if k in self.VEC:
                self.t[k] = torch.full((3, n), float("nan"), dtype=torch.float32, device=device)
            elif k == "uv":
                self.t[k] = torch.full((n, 2), float("nan"), dtype=torch.float32, device=device)
            elif k == "epsilon":
                self.t[k] = torch.full((n,), float("nan"), dtype=torch.float32, device=device)
            elif k in ("front", "intersected"):
                self.t[k] = torch.full((n,), 0xFF, dtype=torch.uint8, device=device)
            else:
                self.t[k] = torch.full((n,), -1, dtype=torch.int32, device=device)

    def __getitem__(self, k):
        return self.t[k]

    def c_struct(self) -> IsectBuffer:
        b = IsectBuffer()
        for k in self.ALL:
            x = self.t.get(k)
            if k in self.VEC:
                arr = getattr(b, k)
                for j in range(3):
                    arr[j] = None if x is None else x[j].data_ptr()
            else:
                setattr(b, k, None if x is None else x.data_ptr())
        return b


def trace_isect(tracer: CudaTracer, scene: DeviceScene, rays, any_hit: bool = True, stencil=None, out=None,
                stream=None, fields=None) -> IntersectionBuffer:
    """CudaTracer::trace(RayBuffer, IntersectionBuffer&, SceneBuffer&, stencil,
    any_hit) (cudatracer.h:87).  Note the reference's default any_hit=True."""
    n = rays.shape[0]
    if out is None:
        out = IntersectionBuffer(n, rays.device, fields)
    b = out.c_struct()
    check(lib().rb2_trace_isect(tracer.handle, scene.handle, _ptr(rays), n, 1 if any_hit else 0, _ptr(stencil),
                                C.byref(b), _stream_handle(stream)))
    return out


FILTER_KINDS = {"none": 0, "box": 1, "triangle": 2, "gaussian": 3}


@dataclass
class Filter:
    """Film reconstruction filter (core/filter.h:46-132): FilterBox,
    FilterTriangle, FilterGaussian(xwidth, ywidth, alpha); "none" = mean of
    the pixel's own samples."""
    kind: str = "none"
    xwidth: float = 0.5
    ywidth: float = 0.5
    alpha: float = 2.0

    def c_struct(self) -> _Filter:
        return _Filter(FILTER_KINDS[self.kind], self.xwidth, self.ywidth, self.alpha)


def filter_table(f: Filter) -> np.ndarray:
    """The film's 16 x 16 precomputed filter table."""
    t = np.zeros(256, np.float32)
    c = f.c_struct()
    check(lib().rb2_filter_table(C.byref(c), _ptr(t)))
    return t.reshape(16, 16)


def film_develop(f: Filter, width: int, height: int, spp: int, xy, L, out=None, stream=None):
    """Filtered image from sample-major samples: xy (spp*w*h, 2) raster
    positions, L (spp*w*h, 4) radiance, device tensors; returns (h*w, 3)."""
    import torch
    if out is None:
        out = torch.empty((width * height, 3), dtype=torch.float32, device=L.device)
    c = f.c_struct()
    check(lib().rb2_film_develop(C.byref(c), width, height, spp, _ptr(xy), _ptr(L), _ptr(out), _stream_handle(stream)))
    return out


def write_pfm(path: str, rgb: np.ndarray, width: int, height: int) -> None:
    """Writes an (h*w, 3) float image, top row first, as a PFM file."""
    rgb = np.ascontiguousarray(rgb, np.float32)
    check(lib().rb2_image_write_pfm(str(path).encode(), _ptr(rgb), width, height))


# Reference-compatibility switches (rb2_render.h): each reproduces one
# behaviour of the reference that the integrators otherwise correct.
COMPAT_AO_DIRECTION, COMPAT_RR_DIVISOR, COMPAT_NEE_RESEED = 1, 2, 4


@dataclass
class AmbientOcclusionIntegratorParams:
    samples: int = 16
    radius: float = 0.1
    seed: int = 7
    compat: int = 0                 # COMPAT_AO_DIRECTION: the reference's AO direction formula


@dataclass
class PathIntegratorParams:
    spp: int = 16
    max_depth: int = 8
    rr_start: int = 3
    rr_prob: float = 0.95
    seed: int = 11
    spp_per_wave: int = 0
    compat: int = 0                 # COMPAT_RR_DIVISOR | COMPAT_NEE_RESEED


BDPT_MODES = {"sk": 0, "mk": 1, "sort": 2}
BDPT_ESTIMATORS = {"unbiased": 0, "reference": 1}


@dataclass
class BidirectionalPathIntegratorLvcParams:
    """The reference's BidirectionalPathIntegratorLvcParams (core/params.h:108-120)
    with its integrator file's names, plus `estimator`: "unbiased" (this
    library's estimator; max_path_length caps the whole path) or "reference"
    (the reference's own estimator: preparation pass, 1 / ((bounce + 1) +
    depth) connection weights, separate light / camera depths; see
    rb2_render.h).  rr_start / rr_prob give both subpaths' Russian roulette
    unless light_path_rrstart / cam_path_rrstart / cam_path_rrprob are set."""
    spp: int = 16
    max_path_length: int = 6
    num_light_paths: int = 0        # 0: one light subpath per pixel per iteration
    connections: int = 1            # m_num_cam_path_connections (reference default 5, config 3: 1)
    rr_start: int = 3
    rr_prob: float = 0.95
    seed: int = 13
    estimator: str = "unbiased"
    num_prep_paths: int = 10000
    num_light_path_max_depth: int = 8
    light_path_rrstart: int | None = None
    num_cam_path_max_depth: int = 8
    cam_path_rrstart: int | None = None
    cam_path_rrprob: float | None = None
    num_cam_path_sample_connections: int = 10
    mode: str = "sk"

    def c_struct(self) -> BdptLvcParams:
        return BdptLvcParams(
            self.spp, self.num_prep_paths, self.num_light_paths, self.num_light_path_max_depth,
            self.rr_start if self.light_path_rrstart is None else self.light_path_rrstart,
            self.num_cam_path_max_depth, self.rr_start if self.cam_path_rrstart is None else self.cam_path_rrstart,
            self.rr_prob if self.cam_path_rrprob is None else self.cam_path_rrprob,
            self.num_cam_path_sample_connections, self.connections, BDPT_MODES[self.mode],
            BDPT_ESTIMATORS[self.estimator], self.max_path_length, 0, self.seed)


# RayCastShade (core/params.h:139-146), by the names the reference's integrator
# file uses (config/configuration.cpp:222-250; "uvs" has no name there).
RAYCAST_SHADES = {"primitive_id": 0, "material_id": 1, "normals": 2, "uvs": 3, "uniform": 4}


@dataclass
class RayCastIntegratorParams:
    shade: str = "primitive_id"     # primitive_id | material_id | normals | uvs | uniform
    spp: int = 1
    seed: int = 5


class Integrator:
    """Binds a tracer and a device scene; owns the wavefront scratch."""

    def __init__(self, tracer: CudaTracer, scene: DeviceScene):
        self.tracer, self.scene = tracer, scene
        self._it = C.c_void_p()
        check(lib().rb2_integrator_create(tracer.handle, scene.handle, C.byref(self._it)))

    def set_launch(self, block_threads: int = 0, regs: int = 0, fetch_threshold: int = 0, node_threshold: int = 0):
        """Launch shape of the integrator's traversal kernels (0 = default)."""
        from ._native import LaunchConfig
        c = LaunchConfig(block_threads, 0, fetch_threshold, regs, node_threshold)
        check(lib().rb2_integrator_set_launch(self._it, C.byref(c)))

    def set_wave(self, paths: int = 0):
        """Paths in flight per wave (0: defaults); see rb2_integrator_set_wave."""
        check(lib().rb2_integrator_set_wave(self._it, int(paths)))

    def set_timing(self, on: bool = True):
        """Time the traversal launches of each render (stats()["trace_ms"])."""
        check(lib().rb2_integrator_set_timing(self._it, 1 if on else 0))

    def set_filter(self, f: "Filter | None"):
        """Film filter of render_pt / render_bdpt / render_raycast (None: per-pixel mean)."""
        if f is None:
            check(lib().rb2_integrator_set_filter(self._it, None))
        else:
            c = f.c_struct()
            check(lib().rb2_integrator_set_filter(self._it, C.byref(c)))

    def __del__(self):
        it = getattr(self, "_it", None)
        if it and it.value and lib is not None:  # lib is None at interpreter shutdown
            lib().rb2_integrator_destroy(it)
            self._it = C.c_void_p()

    def render_ao(self, camera, params: AmbientOcclusionIntegratorParams, out=None, stream=None):
        import torch
        n = camera.width * camera.height
        if out is None:
            out = torch.empty((n,), dtype=torch.float32, device="cuda")
        p = AoParams(params.samples, params.radius, params.seed, params.compat, 0)
        check(lib().rb2_render_ao(self._it, C.byref(camera.c), C.byref(p), _ptr(out), _stream_handle(stream)))
        return out

    def render_pt(self, camera, params: PathIntegratorParams, out=None, stream=None):
        import torch
        n = camera.width * camera.height
        if out is None:
            out = torch.empty((n, 3), dtype=torch.float32, device="cuda")
        p = PtParams(params.spp, params.max_depth, params.rr_start, params.rr_prob, params.seed,
                     params.spp_per_wave, params.compat)
        check(lib().rb2_render_pt(self._it, C.byref(camera.c), C.byref(p), _ptr(out), _stream_handle(stream)))
        return out

    def render_pt_progressive(self, camera, params: PathIntegratorParams, first_sample: int, sums, out=None,
                              stream=None):
        """Adds samples [first_sample, first_sample + params.spp) of every
        pixel to `sums` (a float32 CUDA tensor of 4 values per pixel, zeroed
        before the first call) and returns the image over all samples summed
        so far in `out` (allocated when None).  Unfiltered, any split of the
        samples over calls gives the same image as one render_pt call of the
        total spp (rb2_render_pt_progressive)."""
        import torch
        n = camera.width * camera.height
        if sums.numel() != 4 * n or sums.dtype != torch.float32 or not sums.is_cuda or not sums.is_contiguous():
            raise ValueError("sums must be a contiguous float32 CUDA tensor of 4 values per pixel")
        if out is None:
            out = torch.empty((n, 3), dtype=torch.float32, device="cuda")
        p = PtParams(params.spp, params.max_depth, params.rr_start, params.rr_prob, params.seed,
                     params.spp_per_wave, params.compat)
        check(lib().rb2_render_pt_progressive(self._it, C.byref(camera.c), C.byref(p), int(first_sample), _ptr(sums),
                                              _ptr(out), _stream_handle(stream)))
        return out

    def render_bdpt(self, camera, params: BidirectionalPathIntegratorLvcParams, out=None, stream=None):
        import torch
        n = camera.width * camera.height
        if out is None:
            out = torch.empty((n, 3), dtype=torch.float32, device="cuda")
        p = params.c_struct()
        check(lib().rb2_render_bdpt_lvc(self._it, C.byref(camera.c), C.byref(p), _ptr(out), _stream_handle(stream)))
        return out

    def render_raycast(self, camera, params: RayCastIntegratorParams, out=None, stream=None):
        """IntegratorRayCast::render: (w*h, 3) colours, mean over params.spp samples."""
        import torch
        n = camera.width * camera.height
        if out is None:
            out = torch.empty((n, 3), dtype=torch.float32, device="cuda")
        shade = RAYCAST_SHADES[params.shade] if isinstance(params.shade, str) else int(params.shade)
        p = RayCastParams(params.spp, shade, params.seed)
        check(lib().rb2_render_raycast(self._it, C.byref(camera.c), C.byref(p), _ptr(out), _stream_handle(stream)))
        return out

    def stats(self, stream=None) -> dict:
        s = RenderStats()
        check(lib().rb2_integrator_stats(self._it, C.byref(s), _stream_handle(stream)))
        return {k: getattr(s, k) for k, _ in RenderStats._fields_}

    def device_bytes(self) -> int:
        v = C.c_uint64()
        check(lib().rb2_integrator_device_bytes(self._it, C.byref(v)))
        return v.value
