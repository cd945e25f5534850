"""ctypes bindings for librb2.so (the C ABI declared in include/rb2*.h).

The library is loaded from this package's _lib/ directory.  There is no
fallback: if the shared object is missing, loading raises immediately.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "_lib" / "librb2.so"
_lib = None


class BuildParams(C.Structure):
    """rb2_build_params; field meanings follow Platform / BuildParams of the
    reference (accelerators/sbvh/platform.h:78-90, bvh.h:104-112)."""
    _fields_ = [
        ("sah_node_cost", C.c_float), ("sah_triangle_cost", C.c_float),
        ("min_leaf_size", C.c_uint32), ("max_leaf_size", C.c_uint32),
        ("split_alpha", C.c_float), ("max_depth", C.c_uint32), ("max_spatial_depth", C.c_uint32),
        ("spatial_bins", C.c_uint32), ("object_bins", C.c_uint32), ("exact_sweep_max", C.c_uint32),
        ("num_threads", C.c_int32), ("layout", C.c_uint32),
    ]


class BvhCounts(C.Structure):
    _fields_ = [
        ("n_nodes_u4", C.c_uint64), ("n_woop_u4", C.c_uint64), ("n_triidx", C.c_uint64),
        ("n_inner", C.c_uint32), ("n_leaves", C.c_uint32), ("n_tri_refs", C.c_uint32), ("n_tris", C.c_uint32),
        ("max_depth", C.c_uint32), ("layout", C.c_uint32), ("sah", C.c_float), ("build_ms", C.c_double),
    ]


class Cw8Counts(C.Structure):
    _fields_ = [("n_nodes", C.c_uint32), ("n_tris", C.c_uint32), ("depth", C.c_uint32), ("reserved", C.c_uint32)]


class LaunchConfig(C.Structure):
    _fields_ = [("block_threads", C.c_uint32), ("ctas_per_sm", C.c_uint32),
                ("fetch_threshold", C.c_uint32), ("regs", C.c_uint32), ("node_threshold", C.c_uint32)]


class TraceJob(C.Structure):
    _fields_ = [("tracer", C.c_void_p), ("d_rays", C.c_void_p), ("n", C.c_uint64), ("mode", C.c_uint32),
                ("reserved", C.c_uint32), ("d_mask", C.c_void_p), ("d_out", C.c_void_p)]


class HostJob(C.Structure):
    _fields_ = [("tracer", C.c_void_p), ("h_rays", C.c_void_p), ("n", C.c_uint64), ("mode", C.c_uint32),
                ("reserved", C.c_uint32), ("h_mask", C.c_void_p), ("h_out", C.c_void_p)]


class DevBvh(C.Structure):
    _fields_ = [("nodes", C.c_void_p), ("woop", C.c_void_p), ("triidx", C.c_void_p), ("n_nodes_u4", C.c_uint64),
                ("n_woop_u4", C.c_uint64)]


class DevScene(C.Structure):
    _fields_ = [("verts", C.c_void_p), ("tris", C.c_void_p), ("nv", C.c_uint32), ("ntri", C.c_uint32)]


class IsectBuffer(C.Structure):
    _fields_ = [("position", C.c_void_p * 3), ("geometric_normal", C.c_void_p * 3),
                ("shading_normal", C.c_void_p * 3), ("incoming_direction", C.c_void_p * 3), ("uv", C.c_void_p),
                ("primitive_id", C.c_void_p), ("primitive_material_id", C.c_void_p), ("front", C.c_void_p),
                ("intersected", C.c_void_p), ("epsilon", C.c_void_p)]


class BsdfLayer(C.Structure):
    _fields_ = [("type", C.c_uint32), ("fresnel", C.c_uint32), ("color", C.c_float * 3), ("sigma_deg", C.c_float),
                ("etai", C.c_float), ("etat", C.c_float), ("exponent", C.c_float), ("eta", C.c_float * 3),
                ("k", C.c_float * 3)]


class MaterialDesc(C.Structure):
    _fields_ = [("n_layers", C.c_uint32), ("reserved", C.c_uint32), ("layer", BsdfLayer * 4)]


class Filter(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("xwidth", C.c_float), ("ywidth", C.c_float), ("alpha", C.c_float)]


class BatchConfig(C.Structure):
    _fields_ = [("block_threads", C.c_uint32), ("ctas_per_sm", C.c_uint32), ("fetch_threshold", C.c_uint32),
                ("chunk", C.c_uint32), ("node_order", C.c_uint32), ("regs", C.c_uint32), ("reorder", C.c_uint32),
                ("node_threshold", C.c_uint32)]


class AoParams(C.Structure):
    _fields_ = [("samples", C.c_uint32), ("radius", C.c_float), ("seed", C.c_uint64), ("compat", C.c_uint32),
                ("reserved", C.c_uint32)]


class PtParams(C.Structure):
    _fields_ = [("spp", C.c_uint32), ("max_depth", C.c_uint32), ("rr_start", C.c_uint32), ("rr_prob", C.c_float),
                ("seed", C.c_uint64), ("spp_per_wave", C.c_uint32), ("compat", C.c_uint32)]


class BdptParams(C.Structure):
    _fields_ = [("spp", C.c_uint32), ("max_path_length", C.c_uint32), ("num_light_paths", C.c_uint32),
                ("connections", C.c_uint32), ("rr_start", C.c_uint32), ("rr_prob", C.c_float), ("seed", C.c_uint64)]


class BdptLvcParams(C.Structure):
    """rb2_bdpt_lvc_params: the reference's BidirectionalPathIntegratorLvcParams
    (core/params.h:108-120) plus the estimator choice."""
    _fields_ = [("spp", C.c_uint32), ("num_prep_paths", C.c_uint32), ("num_light_paths", C.c_uint32),
                ("num_light_path_max_depth", C.c_uint32), ("light_path_rrstart", C.c_uint32),
                ("num_cam_path_max_depth", C.c_uint32), ("cam_path_rrstart", C.c_uint32),
                ("cam_path_rrprob", C.c_float), ("num_cam_path_sample_connections", C.c_uint32),
                ("num_cam_path_connections", C.c_uint32), ("mode", C.c_uint32), ("estimator", C.c_uint32),
                ("max_path_length", C.c_uint32), ("reserved", C.c_uint32), ("seed", C.c_uint64)]


class RayCastParams(C.Structure):
    _fields_ = [("spp", C.c_uint32), ("shade", C.c_uint32), ("seed", C.c_uint64)]


class RenderStats(C.Structure):
    _fields_ = [("primary_rays", C.c_uint64), ("extension_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("connection_rays", C.c_uint64), ("light_rays", C.c_uint64), ("lvc_vertices", C.c_uint64),
                ("trace_ms", C.c_double)]


class Camera(C.Structure):
    _fields_ = [
        ("raster_to_camera", C.c_float * 16), ("camera_to_world", C.c_float * 16),
        ("width", C.c_uint32), ("height", C.c_uint32),
        ("eye", C.c_float * 3), ("lookat", C.c_float * 3), ("up", C.c_float * 3), ("fov_deg", C.c_float),
    ]


P = C.c_void_p
U32 = C.c_uint32
U64 = C.c_uint64
I32 = C.c_int

# name -> (restype, argtypes)
SIGNATURES = {
    "rb2_last_error": (C.c_char_p, []),
    "rb2_version": (C.c_char_p, []),
    "rb2_build_params_default": (C.c_int, [C.POINTER(BuildParams)]),
    "rb2_bvh_build": (C.c_int, [P, U32, P, U32, C.POINTER(BuildParams), C.POINTER(P)]),
    "rb2_bvh_from_buffers": (C.c_int, [P, U64, P, U64, P, U64, C.POINTER(P)]),
    "rb2_bvh_counts_get": (C.c_int, [P, C.POINTER(BvhCounts)]),
    "rb2_bvh_nodes": (P, [P]),
    "rb2_bvh_woop": (P, [P]),
    "rb2_bvh_triidx": (P, [P]),
    "rb2_host_bvh_free": (None, [P]),
    "rb2_bvh_save": (C.c_int, [P, C.c_char_p]),
    "rb2_bvh_save_text": (C.c_int, [P, C.c_char_p]),
    "rb2_bvh_load": (C.c_int, [C.c_char_p, C.POINTER(P)]),
    "rb2_tracer_create": (C.c_int, [P, C.POINTER(P)]),
    "rb2_tracer_destroy": (C.c_int, [P]),
    "rb2_tracer_set_launch": (C.c_int, [P, C.POINTER(LaunchConfig)]),
    "rb2_tracer_device_bytes": (C.c_int, [P, C.POINTER(U64)]),
    "rb2_trace": (C.c_int, [P, P, U32, I32, P, P, P]),
    "rb2_trace_host": (C.c_int, [P, P, U32, I32, P, P, P]),
    "rb2_trace_occlusion": (C.c_int, [P, P, U32, P, P, P]),
    "rb2_tracer_status": (C.c_int, [P, C.POINTER(U32), P]),
    "rb2_tracer_set_node_order": (C.c_int, [P, U32]),
    "rb2_integrator_set_wave": (C.c_int, [P, C.c_uint64]),
    "rb2_tracer_get_node_order": (C.c_int, [P, C.POINTER(U32)]),
    "rb2_bvh_cw8_layout": (C.c_int, [P, C.POINTER(Cw8Counts), P, P, P]),
    "rb2_tracer_dev_bvh": (C.c_int, [P, C.POINTER(DevBvh)]),
    "rb2_trace_per_thread": (C.c_int, [P, P, U32, I32, P, P, P]),
    "rb2_scene_dev_view": (C.c_int, [P, C.POINTER(DevScene)]),
    "rb2_trace_isect": (C.c_int, [P, P, P, U32, I32, P, C.POINTER(IsectBuffer), P]),
    "rb2_filter_table": (C.c_int, [C.POINTER(Filter), P]),
    "rb2_scene_set_materials": (C.c_int, [P, C.POINTER(MaterialDesc), U32]),
    "rb2_integrator_set_launch": (C.c_int, [P, C.POINTER(LaunchConfig)]),
    "rb2_integrator_set_timing": (C.c_int, [P, I32]),
    "rb2_material_query": (C.c_int, [P, I32, P, P, U32, P, P]),
    "rb2_film_develop": (C.c_int, [C.POINTER(Filter), U32, U32, U32, P, P, P, P]),
    "rb2_image_write_pfm": (C.c_int, [C.c_char_p, P, U32, U32]),
    "rb2_integrator_set_filter": (C.c_int, [P, C.POINTER(Filter)]),
    "rb2_pipeline_create": (C.c_int, [U64, U32, C.POINTER(P)]),
    "rb2_pipeline_destroy": (C.c_int, [P]),
    "rb2_trace_host_jobs": (C.c_int, [P, C.POINTER(HostJob), U32, P]),
    "rb2_batch_create": (C.c_int, [C.POINTER(TraceJob), U32, C.POINTER(P)]),
    "rb2_batch_destroy": (C.c_int, [P]),
    "rb2_batch_set_config": (C.c_int, [P, C.POINTER(BatchConfig)]),
    "rb2_batch_get_config": (C.c_int, [P, C.POINTER(BatchConfig)]),
    "rb2_batch_launch": (C.c_int, [P, P]),
    "rb2_batch_capture": (C.c_int, [P, P]),
    "rb2_batch_status": (C.c_int, [P, C.POINTER(U32), P]),
    "rb2_batch_autotune": (C.c_int, [P, P, U32, C.POINTER(BatchConfig), C.POINTER(C.c_double)]),
    "rb2_scene_create": (C.c_int, [P, U32, P, U32, P, U32, P, P, C.POINTER(P)]),
    "rb2_scene_destroy": (C.c_int, [P]),
    "rb2_scene_device_bytes": (C.c_int, [P, C.POINTER(U64)]),
    "rb2_integrator_create": (C.c_int, [P, P, C.POINTER(P)]),
    "rb2_integrator_destroy": (C.c_int, [P]),
    "rb2_integrator_device_bytes": (C.c_int, [P, C.POINTER(U64)]),
    "rb2_integrator_stats": (C.c_int, [P, C.POINTER(RenderStats), P]),
    "rb2_render_ao": (C.c_int, [P, C.POINTER(Camera), C.POINTER(AoParams), P, P]),
    "rb2_render_pt": (C.c_int, [P, C.POINTER(Camera), C.POINTER(PtParams), P, P]),
    "rb2_render_pt_progressive": (C.c_int, [P, C.POINTER(Camera), C.POINTER(PtParams), C.c_uint32, P, P, P]),
    "rb2_render_raycast": (C.c_int, [P, C.POINTER(Camera), C.POINTER(RayCastParams), P, P]),
    "rb2_render_bdpt": (C.c_int, [P, C.POINTER(Camera), C.POINTER(BdptParams), P, P]),
    "rb2_render_bdpt_lvc": (C.c_int, [P, C.POINTER(Camera), C.POINTER(BdptLvcParams), P, P]),
    "rb2_camera_init": (C.c_int, [C.POINTER(Camera), P, P, P, U32, U32, C.c_float]),
    "rb2_camera_rays": (C.c_int, [C.POINTER(Camera), U32, U64, I32, P, P]),
    "rb2_camera_rays_at": (C.c_int, [C.POINTER(Camera), P, U32, P, P]),
    "rb2_gen_heightfield_counts": (C.c_int, [U32, U32, C.POINTER(U32), C.POINTER(U32)]),
    "rb2_gen_heightfield": (C.c_int, [U64, U32, C.c_float, U32, C.c_float, C.c_float, P, P]),
    "rb2_gen_room_counts": (C.c_int, [U32, U32, U32, U32, C.POINTER(U32), C.POINTER(U32)]),
    "rb2_gen_room": (C.c_int, [U64, U32, U32, U32, C.c_float, C.c_float, U32, P, P, P]),
    "rb2_gen_surface_rays": (C.c_int, [P, U32, P, U32, U64, U64, C.c_float, C.c_float, P, P]),
    "rb2_pcg32_fill": (C.c_int, [U64, U64, U32, P]),
}


class Rb2Error(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"rb2 error {code}: {msg}")
        self.code = code


def lib() -> C.CDLL:
    """Returns the loaded librb2 (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            raise RuntimeError(f"librb2.so not built at {_LIB_PATH}; run `python -m renderbox2_b200.build`")
        L = C.CDLL(str(_LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != 0:
        msg = lib().rb2_last_error()
        raise Rb2Error(rc, msg.decode() if msg else "")
