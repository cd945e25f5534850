"""Python mirror of the reference's scene / BVH / tracer interface.

Names and argument meanings follow renderbox2:
  Scene.add_mesh                core/scene.cpp:83-123
  Platform, BVH.BuildParams     accelerators/sbvh/platform.h:78-90, bvh.h:104-112
  BVH(scene, platform, params)  accelerators/sbvh/bvh.h:115
  CudaBvh(bvh) / CudaBvh(path)  accelerators/sbvh/cudabvh.h:80-98
  CudaTracer(bvh).trace(...)    accelerators/sbvh/cudatracer.h:67-101
Every call goes through librb2's C ABI; errors raise Rb2Error.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from ._native import BuildParams as _BuildParams
from ._native import BvhCounts, Cw8Counts, LaunchConfig, check, lib


def _ptr(a) -> int:
    """Address of a contiguous numpy array or torch tensor."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
        return a.ctypes.data
    assert a.is_contiguous(), "tensor must be contiguous"
    return a.data_ptr()


def _stream_handle(stream) -> int:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


# ------------------------------------------------------------------------ scene
class Scene:
    """Host triangle soup.  Meshes are concatenated; every triangle of an
    emissive mesh becomes a light (core/scene.cpp:105-113)."""

    def __init__(self):
        self.vertices = np.zeros((0, 3), np.float32)
        self.indices = np.zeros((0, 3), np.uint32)
        self.material_ids = np.zeros((0,), np.uint32)
        self.light_ids_to_primitive_ids = np.zeros((0,), np.uint32)

    @property
    def num_triangles(self) -> int:
        return int(self.indices.shape[0])

    @property
    def num_lights(self) -> int:
        return int(self.light_ids_to_primitive_ids.shape[0])

    def add_mesh(self, vertices, indices, material_ids=0, is_emissive=False):
        v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
        i = np.ascontiguousarray(indices, np.uint32).reshape(-1, 3)
        base_v, base_t = self.vertices.shape[0], self.indices.shape[0]
        m = np.broadcast_to(np.asarray(material_ids, np.uint32), (i.shape[0],)).copy()
        self.vertices = np.concatenate([self.vertices, v])
        self.indices = np.concatenate([self.indices, i + np.uint32(base_v)])
        self.material_ids = np.concatenate([self.material_ids, m])
        if is_emissive:
            self.light_ids_to_primitive_ids = np.concatenate(
                [self.light_ids_to_primitive_ids, np.arange(base_t, base_t + i.shape[0], dtype=np.uint32)])
        return self

    def bounds(self):
        return self.vertices.min(axis=0), self.vertices.max(axis=0)


# -------------------------------------------------------------------------- BVH
@dataclass
class Platform:
    """SAH costs and leaf-size limits (accelerators/sbvh/platform.h:78-90)."""
    sah_node_cost: float = 1.0
    sah_triangle_cost: float = 1.0
    min_leaf_size: int = 1
    max_leaf_size: int = 0x7FFFFFF


@dataclass
class BuildParams:
    """Builder knobs; split_alpha as bvh.h:110, the rest are this builder's."""
    split_alpha: float = 1.0e-5
    max_depth: int = 64
    max_spatial_depth: int = 48
    spatial_bins: int = 64
    object_bins: int = 64
    exact_sweep_max: int = 512
    num_threads: int = 0
    stats: dict = field(default_factory=dict)


class BVH:
    """SBVH over a Scene, already packed to the Compact2 device layout."""

    def __init__(self, scene: Scene, platform: Platform | None = None, params: BuildParams | None = None,
                 _handle=None):
        L = lib()
        self._h = C.c_void_p()
        self.scene = scene
        if _handle is not None:
            self._h = _handle
        else:
            platform = platform or Platform()
            params = params or BuildParams()
            p = _BuildParams()
            check(L.rb2_build_params_default(C.byref(p)))
            p.sah_node_cost = platform.sah_node_cost
            p.sah_triangle_cost = platform.sah_triangle_cost
            p.min_leaf_size = platform.min_leaf_size
            p.max_leaf_size = platform.max_leaf_size
            p.split_alpha = params.split_alpha
            p.max_depth = params.max_depth
            p.max_spatial_depth = params.max_spatial_depth
            p.spatial_bins = params.spatial_bins
            p.object_bins = params.object_bins
            p.exact_sweep_max = params.exact_sweep_max
            p.num_threads = params.num_threads
            v = np.ascontiguousarray(scene.vertices, np.float32)
            i = np.ascontiguousarray(scene.indices, np.uint32)
            check(L.rb2_bvh_build(_ptr(v), v.shape[0], _ptr(i), i.shape[0], C.byref(p), C.byref(self._h)))
            params.stats.update(self.stats())

    @classmethod
    def from_buffers(cls, nodes, woop, triidx, scene: Scene | None = None) -> "BVH":
        nodes = np.ascontiguousarray(nodes, np.uint32).reshape(-1, 4)
        woop = np.ascontiguousarray(woop, np.uint32).reshape(-1, 4)
        triidx = np.ascontiguousarray(triidx, np.uint32).reshape(-1)
        h = C.c_void_p()
        check(lib().rb2_bvh_from_buffers(_ptr(nodes), nodes.shape[0], _ptr(woop), woop.shape[0], _ptr(triidx),
                                         triidx.shape[0], C.byref(h)))
        return cls(scene, _handle=h)

    @classmethod
    def load(cls, path: str, scene: Scene | None = None) -> "BVH":
        h = C.c_void_p()
        check(lib().rb2_bvh_load(str(path).encode(), C.byref(h)))
        return cls(scene, _handle=h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and h.value and lib is not None:  # lib is None at interpreter shutdown
            lib().rb2_host_bvh_free(h)
            self._h = C.c_void_p()

    @property
    def handle(self):
        return self._h

    def counts(self) -> BvhCounts:
        c = BvhCounts()
        check(lib().rb2_bvh_counts_get(self._h, C.byref(c)))
        return c

    def stats(self) -> dict:
        c = self.counts()
        return {k: getattr(c, k) for k, _ in BvhCounts._fields_}

    def _buf(self, getter, n, cols, copy=True):
        ptr = getter(self._h)
        if n == 0:
            return np.zeros((0, cols) if cols > 1 else (0,), np.uint32)
        arr = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_uint32)), shape=(n * cols,))
        if copy:
            arr = arr.copy()
        return arr.reshape(-1, cols) if cols > 1 else arr

    def buffers_view(self):
        """Zero-copy (nodes, woop, triidx) views; valid while this BVH lives."""
        c = self.counts()
        L = lib()
        return (self._buf(L.rb2_bvh_nodes, c.n_nodes_u4, 4, False), self._buf(L.rb2_bvh_woop, c.n_woop_u4, 4, False),
                self._buf(L.rb2_bvh_triidx, c.n_triidx, 1, False))

    # CudaBvh getters (cudabvh.h:95-97)
    def get_node_buffer(self) -> np.ndarray:
        return self._buf(lib().rb2_bvh_nodes, self.counts().n_nodes_u4, 4)

    def get_tri_woop_buffer(self) -> np.ndarray:
        return self._buf(lib().rb2_bvh_woop, self.counts().n_woop_u4, 4)

    def get_tri_index_buffer(self) -> np.ndarray:
        return self._buf(lib().rb2_bvh_triidx, self.counts().n_triidx, 1)

    def cw8_layout(self) -> dict:
        """The compressed 8-wide layout the tracer builds for NODE_ORDER_CW8:
        nodes (n, 20) uint32 words, woop (n_tris, 12) uint32 Woop rows, triidx
        (n_tris,) original triangle ids, depth (wide levels)."""
        c = Cw8Counts()
        check(lib().rb2_bvh_cw8_layout(self._h, C.byref(c), None, None, None))
        nodes = np.zeros((c.n_nodes, 20), np.uint32)
        woop = np.zeros((c.n_tris, 12), np.uint32)
        tri = np.zeros((c.n_tris,), np.uint32)
        check(lib().rb2_bvh_cw8_layout(self._h, C.byref(c), _ptr(nodes), _ptr(woop), _ptr(tri)))
        return {"nodes": nodes, "woop": woop, "triidx": tri, "depth": int(c.depth)}

    def serialize(self, path: str) -> None:
        check(lib().rb2_bvh_save(self._h, str(path).encode()))

    def serialize_text(self, path: str) -> None:
        check(lib().rb2_bvh_save_text(self._h, str(path).encode()))


CudaBvh = BVH  # the packed layout is produced together with the tree


# ----------------------------------------------------------------------- tracer
class CudaTracer:
    """Device-resident BVH plus the bulk traversal entry points."""

    def __init__(self, bvh: BVH):
        self.bvh = bvh
        self._t = C.c_void_p()
        check(lib().rb2_tracer_create(bvh.handle, C.byref(self._t)))

    def __del__(self):
        t = getattr(self, "_t", None)
        if t and t.value and lib is not None:  # lib is None at interpreter shutdown
            lib().rb2_tracer_destroy(t)
            self._t = C.c_void_p()

    @property
    def handle(self):
        return self._t

    def device_bytes(self) -> int:
        v = C.c_uint64()
        check(lib().rb2_tracer_device_bytes(self._t, C.byref(v)))
        return v.value

    def set_launch(self, ctas_per_sm=0, fetch_threshold=0, block_threads=0, regs=0, node_threshold=0):
        """Launch shape of this tracer's bulk traversals (rb2_launch_config;
        0 = the tuned default for each field)."""
        cfg = LaunchConfig(block_threads, ctas_per_sm, fetch_threshold, regs, node_threshold)
        check(lib().rb2_tracer_set_launch(self._t, C.byref(cfg)))

    def set_node_order(self, order: int):
        """Node layout of the bulk traversals: NODE_ORDER_DFS (the Compact2
        buffer as built), NODE_ORDER_BFS, NODE_ORDER_WIDE4 or NODE_ORDER_CW8.
        Integrators traverse the compressed 8-wide layout when it is set, the
        binary buffer otherwise."""
        check(lib().rb2_tracer_set_node_order(self._t, int(order)))

    def node_order(self) -> int:
        v = C.c_uint32()
        check(lib().rb2_tracer_get_node_order(self._t, C.byref(v)))
        return v.value

    def trace(self, rays, any_hit: bool = False, stencil=None, out=None, stream=None):
        """rays: CUDA float32 tensor (n, 8).  Returns an int32 tensor (n, 4) of
        (prim, t bits, u bits, v bits); see hits_view()."""
        import torch
        n = rays.shape[0]
        if out is None:
            out = torch.empty((n, 4), dtype=torch.int32, device=rays.device)
        check(lib().rb2_trace(self._t, _ptr(rays), n, 1 if any_hit else 0, _ptr(stencil), _ptr(out),
                              _stream_handle(stream)))
        return out

    def trace_occlusion(self, rays, stencil=None, out=None, stream=None):
        import torch
        n = rays.shape[0]
        if out is None:
            out = torch.empty((n,), dtype=torch.uint8, device=rays.device)
        check(lib().rb2_trace_occlusion(self._t, _ptr(rays), n, _ptr(stencil), _ptr(out), _stream_handle(stream)))
        return out

    def trace_host(self, rays: np.ndarray, any_hit: bool = False, stencil: np.ndarray | None = None,
                   out: np.ndarray | None = None, stream=None) -> np.ndarray:
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        if out is None:
            out = np.empty((n, 4), np.int32)
        check(lib().rb2_trace_host(self._t, _ptr(rays), n, 1 if any_hit else 0, _ptr(stencil), _ptr(out),
                                   _stream_handle(stream)))
        return out

    def trace_per_thread(self, rays, any_hit: bool = False, stencil=None, out=None, stream=None):
        """One thread per ray through the header-only device traversal
        (rb2_device.cuh): the pattern of kernels that trace in their own code."""
        import torch
        n = rays.shape[0]
        if out is None:
            out = torch.empty((n, 4), dtype=torch.int32, device=rays.device)
        check(lib().rb2_trace_per_thread(self._t, _ptr(rays), n, 1 if any_hit else 0, _ptr(stencil), _ptr(out),
                                         _stream_handle(stream)))
        return out

    def get_bvh(self) -> dict:
        """Device view of the BVH (CudaTracer::get_bvh, cudatracer.h:89-101)."""
        from ._native import DevBvh
        d = DevBvh()
        check(lib().rb2_tracer_dev_bvh(self._t, C.byref(d)))
        return {k: getattr(d, k) for k, _ in DevBvh._fields_}

    def status(self, stream=None) -> int:
        v = C.c_uint32()
        check(lib().rb2_tracer_status(self._t, C.byref(v), _stream_handle(stream)))
        return v.value


def hits_view(hits):
    """Splits an (n, 4) int32 hit array into (prim int32, t, u, v float32)."""
    if isinstance(hits, np.ndarray):
        f = hits.view(np.float32)
        return hits[:, 0], f[:, 1], f[:, 2], f[:, 3]
    import torch
    f = hits.view(torch.float32)
    return hits[:, 0], f[:, 1], f[:, 2], f[:, 3]


MODE_CLOSEST, MODE_ANY, MODE_OCCLUSION = 0, 1, 2
NODE_ORDER_DFS, NODE_ORDER_BFS, NODE_ORDER_WIDE4, NODE_ORDER_CW8 = 0, 1, 2, 3


class TraceBatch:
    """Many (scene, ray batch, mode) jobs served by ONE persistent launch.

    jobs: iterable of (tracer, rays tensor (n,8), mode, out tensor, mask or None).
    Buffers are borrowed: keep them alive while the batch exists."""

    def __init__(self, jobs):
        from ._native import TraceJob
        jobs = list(jobs)
        arr = (TraceJob * max(1, len(jobs)))()
        self._keep = []
        for k, (tr, rays, mode, out, mask) in enumerate(jobs):
            arr[k].tracer = tr.handle.value
            arr[k].d_rays = _ptr(rays)
            arr[k].n = int(rays.shape[0])
            arr[k].mode = int(mode)
            arr[k].d_mask = _ptr(mask)
            arr[k].d_out = _ptr(out)
            self._keep.append((tr, rays, out, mask))
        self._b = C.c_void_p()
        check(lib().rb2_batch_create(arr, len(jobs), C.byref(self._b)))

    def __del__(self):
        b = getattr(self, "_b", None)
        if b and b.value and lib is not None:  # lib is None at interpreter shutdown
            lib().rb2_batch_destroy(b)
            self._b = C.c_void_p()

    def config(self) -> dict:
        from ._native import BatchConfig
        c = BatchConfig()
        check(lib().rb2_batch_get_config(self._b, C.byref(c)))
        return {k: getattr(c, k) for k, _ in BatchConfig._fields_}

    def set_config(self, **kw):
        from ._native import BatchConfig
        c = BatchConfig()
        check(lib().rb2_batch_get_config(self._b, C.byref(c)))
        for k, v in kw.items():
            setattr(c, k, v)
        check(lib().rb2_batch_set_config(self._b, C.byref(c)))

    def launch(self, stream=None):
        check(lib().rb2_batch_launch(self._b, _stream_handle(stream)))

    def capture(self, stream):
        check(lib().rb2_batch_capture(self._b, _stream_handle(stream)))

    def autotune(self, stream=None, reps=3):
        from ._native import BatchConfig
        c = BatchConfig()
        ms = C.c_double()
        check(lib().rb2_batch_autotune(self._b, _stream_handle(stream), reps, C.byref(c), C.byref(ms)))
        return {k: getattr(c, k) for k, _ in BatchConfig._fields_}, ms.value

    def status(self, stream=None) -> int:
        v = C.c_uint32()
        check(lib().rb2_batch_status(self._b, C.byref(v), _stream_handle(stream)))
        return v.value


class HostPipeline:
    """Host-buffer traces of many jobs with copies overlapped with traversal.

    Each job's rays are cut into chunks of `chunk_rays` that cycle through
    `depth` CUDA streams: the upload of one chunk, the traversal of another
    and the download of a third run at once.  Use pinned host memory (torch
    `pin_memory()` tensors) for the copies to be asynchronous.

    jobs: iterable of (tracer, host rays (n, 8) float32, mode, host out, mask
    or None); out is (n, 4) int32 for MODE_CLOSEST / MODE_ANY and (n,) uint8
    for MODE_OCCLUSION.  trace_jobs returns when every output is on the host."""

    def __init__(self, chunk_rays: int = 1 << 20, depth: int = 4):
        self._p = C.c_void_p()
        check(lib().rb2_pipeline_create(int(chunk_rays), int(depth), C.byref(self._p)))

    def __del__(self):
        p = getattr(self, "_p", None)
        if p and p.value and lib is not None:  # lib is None at interpreter shutdown
            lib().rb2_pipeline_destroy(p)
            self._p = C.c_void_p()

    @staticmethod
    def job_array(jobs):
        from ._native import HostJob
        jobs = list(jobs)
        arr = (HostJob * max(1, len(jobs)))()
        for k, (tr, rays, mode, out, mask) in enumerate(jobs):
            arr[k].tracer = tr.handle.value
            arr[k].h_rays = _ptr(rays)
            arr[k].n = int(rays.shape[0])
            arr[k].mode = int(mode)
            arr[k].h_mask = _ptr(mask)
            arr[k].h_out = _ptr(out)
        return arr, len(jobs)

    def trace_jobs(self, jobs, stream=None):
        """jobs: a list of tuples as above, or the result of job_array().  The
        work is ordered after `stream` (default: the current torch stream)
        and `stream` waits for it."""
        arr, n = jobs if isinstance(jobs, tuple) else self.job_array(jobs)
        check(lib().rb2_trace_host_jobs(self._p, arr, n, _stream_handle(stream)))
