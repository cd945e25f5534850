"""TEST INFRASTRUCTURE ONLY: the oracle.

Two checkers, both CPU-only, used by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py -- never by the product library:

* ``ref_*``: the reference's own host code (SBVH builder, Compact2 packer,
  text BVH cache, perspective camera, Moller-Trumbore test) compiled in place
  from the reference sources into oracle/_ref/librb2ref.so (oracle/Makefile).
* ``trace`` / ``woop_test`` / ``bruteforce``: the CPU restatement of the
  reference's traversal (oracle/rb2_oracle.c).
* ``isect``: the intersection record of a hit (same file).
* ``filter_table`` / ``film``: the film's filtered reconstruction (same file).
* ``ao`` / ``pt`` / ``bdpt``: FP64 CPU restatements of the integrators
  (same file), scalar per pixel, used as statistical references.

Parity is pinned by comparing the restatement with the reference's own
compiled code and against fixtures in tests/golden/ generated from it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_SO = HERE / "_ref" / "librb2ref.so"
ORACLE_SO = HERE / "liboracle.so"

# The reference checkout is located by oracle/Makefile (override: RB2_REF_SRC).

_ref = None
_orc = None


class RefBvh(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_uint32), ("n_woop", C.c_uint32), ("n_triidx", C.c_uint32), ("layout", C.c_uint32),
        ("nodes", C.POINTER(C.c_uint32)), ("woop", C.POINTER(C.c_uint32)), ("triidx", C.POINTER(C.c_uint32)),
        ("sah", C.c_float), ("n_inner", C.c_uint32), ("n_leaves", C.c_uint32), ("n_tri_refs", C.c_uint32),
        ("build_ms", C.c_double),
    ]


class Hit(C.Structure):
    _fields_ = [("prim", C.c_int32), ("t", C.c_float), ("u", C.c_float), ("v", C.c_float)]


HIT_DTYPE = np.dtype([("prim", np.int32), ("t", np.float32), ("u", np.float32), ("v", np.float32)])
COUNT_DTYPE = np.dtype([("nodes", np.uint32), ("tris", np.uint32), ("leafterms", np.uint32), ("pad", np.uint32)])


def build(ref: bool = True) -> None:
    """Builds liboracle.so, and librb2ref.so when the reference sources exist."""
    targets = ["oracle"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", str(HERE), *targets], check=True)


def have_ref() -> bool:
    return REF_SO.exists()


def ref_lib():
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            raise RuntimeError(f"{REF_SO} not built (make -C oracle ref)")
        L = C.CDLL(str(REF_SO))
        L.rb2ref_build.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_int, C.c_char_p,
                                   C.POINTER(RefBvh)]
        L.rb2ref_build.restype = C.c_int
        L.rb2ref_load.argtypes = [C.c_char_p, C.POINTER(RefBvh)]
        L.rb2ref_load.restype = C.c_int
        L.rb2ref_free.argtypes = [C.POINTER(RefBvh)]
        L.rb2ref_free.restype = None
        L.rb2ref_camera_rays.argtypes = [C.c_void_p] * 3 + [C.c_float] * 3 + [C.c_void_p, C.c_uint32, C.c_void_p]
        L.rb2ref_camera_rays.restype = C.c_int
        L.rb2ref_intersect_triangle.argtypes = [C.c_void_p] * 5
        L.rb2ref_intersect_triangle.restype = C.c_int
        L.rb2ref_normal_and_point.argtypes = [C.c_void_p] * 4 + [C.c_float, C.c_void_p, C.c_void_p]
        L.rb2ref_normal_and_point.restype = C.c_int
        _ref = L
    return _ref


def orc_lib():
    global _orc
    if _orc is None:
        if not ORACLE_SO.exists():
            raise RuntimeError(f"{ORACLE_SO} not built (make -C oracle oracle)")
        L = C.CDLL(str(ORACLE_SO))
        L.rb2o_trace.argtypes = [C.c_void_p] * 4 + [C.c_uint32, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.rb2o_trace.restype = None
        L.rb2o_woop_test.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_void_p]
        L.rb2o_woop_test.restype = C.c_int
        L.rb2o_bruteforce.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_int]
        L.rb2o_bruteforce.restype = None
        L.rb2o_tie_count_brute.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p,
                                           C.c_void_p, C.c_int]
        L.rb2o_tie_count_brute.restype = None
        L.rb2o_tie_count.argtypes = [C.c_void_p] * 4 + [C.c_uint32, C.c_void_p, C.c_void_p, C.c_int]
        L.rb2o_tie_count.restype = None
        L.rb2o_gen_heightfield_counts.argtypes = [C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32),
                                                  C.POINTER(C.c_uint32)]
        L.rb2o_gen_heightfield_counts.restype = C.c_int
        L.rb2o_gen_heightfield.argtypes = [C.c_uint64, C.c_uint32, C.c_float, C.c_uint32, C.c_float, C.c_float,
                                           C.c_void_p, C.c_void_p]
        L.rb2o_gen_heightfield.restype = C.c_int
        L.rb2o_gen_surface_rays.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint64,
                                            C.c_float, C.c_float, C.c_void_p, C.c_void_p]
        L.rb2o_gen_surface_rays.restype = C.c_int
        _orc = L
    return _orc


def _p(a):
    return None if a is None else a.ctypes.data


def _copy_ref(b: RefBvh) -> dict:
    nodes = np.ctypeslib.as_array(b.nodes, shape=(b.n_nodes * 4,)).copy().reshape(-1, 4)
    woop = np.ctypeslib.as_array(b.woop, shape=(b.n_woop * 4,)).copy().reshape(-1, 4)
    triidx = np.ctypeslib.as_array(b.triidx, shape=(b.n_triidx,)).copy()
    return dict(nodes=nodes, woop=woop, triidx=triidx, sah=float(b.sah), n_inner=int(b.n_inner),
                n_leaves=int(b.n_leaves), n_tri_refs=int(b.n_tri_refs), build_ms=float(b.build_ms),
                layout=int(b.layout))


def ref_build(vertices, indices, cache_path: str | None = None) -> dict:
    """The reference SBVH + Compact2 buffers for a triangle soup."""
    v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
    i = np.ascontiguousarray(indices, np.uint32).reshape(-1, 3)
    b = RefBvh()
    rc = ref_lib().rb2ref_build(_p(v), v.shape[0], _p(i), i.shape[0], 1,
                                cache_path.encode() if cache_path else None, C.byref(b))
    if rc != 0:
        raise RuntimeError(f"reference build failed ({rc})")
    try:
        return _copy_ref(b)
    finally:
        ref_lib().rb2ref_free(C.byref(b))


def ref_load(path: str) -> dict:
    b = RefBvh()
    rc = ref_lib().rb2ref_load(str(path).encode(), C.byref(b))
    if rc != 0:
        raise RuntimeError(f"reference cache load failed ({rc})")
    try:
        return _copy_ref(b)
    finally:
        ref_lib().rb2ref_free(C.byref(b))


def ref_camera_rays(eye, lookat, up, width, height, fov, raster_xy) -> np.ndarray:
    xy = np.ascontiguousarray(raster_xy, np.float32).reshape(-1, 2)
    out = np.empty((xy.shape[0], 8), np.float32)
    e, l_, u = (np.asarray(x, np.float32) for x in (eye, lookat, up))
    ref_lib().rb2ref_camera_rays(_p(e), _p(l_), _p(u), float(width), float(height), float(fov), _p(xy),
                                 xy.shape[0], _p(out))
    return out


def ref_intersect_triangle(v0, v1, v2, ray8):
    a = [np.ascontiguousarray(x, np.float32) for x in (v0, v1, v2, ray8)]
    uvt = np.zeros(3, np.float32)
    hit = ref_lib().rb2ref_intersect_triangle(_p(a[0]), _p(a[1]), _p(a[2]), _p(a[3]), _p(uvt))
    return bool(hit), uvt


def ref_normal_and_point(v0, v1, v2, ray8, t):
    """The reference's compute_normal(v0, v1, v2) and Ray(o, d)(t)."""
    a = [np.ascontiguousarray(x, np.float32) for x in (v0, v1, v2, ray8)]
    ng, pt = np.zeros(3, np.float32), np.zeros(3, np.float32)
    ref_lib().rb2ref_normal_and_point(_p(a[0]), _p(a[1]), _p(a[2]), _p(a[3]), float(t), _p(ng), _p(pt))
    return ng, pt


class _IsectSoa(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("position", "ng", "ns", "wi", "uv", "prim", "material", "front",
                                          "intersected", "epsilon")]


def isect(verts, tris4, rays, hits):
    """Intersection records of closest hits (rb2o_isect): a dict of SoA arrays
    position/ng/ns/wi (3, n) float32, uv (n, 2), prim, material (n,) uint32,
    front, intersected (n,) uint8, epsilon (n,) float32.  Fields of missed
    rays keep their initial value (NaN / 0xFFFFFFFF / 0xFF)."""
    verts = np.ascontiguousarray(verts, np.float32)
    tris4 = np.ascontiguousarray(tris4, np.uint32)
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    hits = np.ascontiguousarray(hits, HIT_DTYPE)
    n = rays.shape[0]
    out = {k: np.full((3, n), np.nan, np.float32) for k in ("position", "ng", "ns", "wi")}
    out["uv"] = np.full((n, 2), np.nan, np.float32)
    out["prim"] = np.full(n, 0xFFFFFFFF, np.uint32)
    out["material"] = np.full(n, 0xFFFFFFFF, np.uint32)
    out["front"] = np.full(n, 0xFF, np.uint8)
    out["intersected"] = np.full(n, 0xFF, np.uint8)
    out["epsilon"] = np.full(n, np.nan, np.float32)
    soa = _IsectSoa(**{k: _p(v) for k, v in out.items()})
    L = orc_lib()
    L.rb2o_isect.argtypes = [C.c_void_p] * 4 + [C.c_uint32, C.POINTER(_IsectSoa)]
    L.rb2o_isect.restype = None
    L.rb2o_isect(_p(verts), _p(tris4), _p(rays), _p(hits), n, C.byref(soa))
    return out


RAY_TYPES = ("camera", "extension", "shadow", "connection", "light")


def counts_reset(on: bool = True) -> None:
    """Starts (or stops) the integrator references' per-ray-type visit counts."""
    L = orc_lib()
    L.rb2o_counts_reset.argtypes = [C.c_int]
    L.rb2o_counts_reset.restype = None
    L.rb2o_counts_reset(1 if on else 0)


def counts_read() -> dict:
    """{ray type: {nodes, tris, leafterms, rays}} accumulated since counts_reset."""
    L = orc_lib()
    L.rb2o_counts_read.argtypes = [C.c_void_p]
    L.rb2o_counts_read.restype = None
    out = np.zeros((len(RAY_TYPES), 4), np.uint64)
    L.rb2o_counts_read(out.ctypes.data)
    return {t: dict(zip(("nodes", "tris", "leafterms", "rays"), (int(x) for x in out[i])))
            for i, t in enumerate(RAY_TYPES)}


FILTER_KINDS = {"none": 0, "box": 1, "triangle": 2, "gaussian": 3}


def filter_table(kind: str, xwidth: float, ywidth: float, alpha: float = 0.0) -> np.ndarray:
    """The film's 16 x 16 filter table (rb2o_filter_table)."""
    L = orc_lib()
    L.rb2o_filter_table.argtypes = [C.c_uint32, C.c_float, C.c_float, C.c_float, C.c_void_p]
    L.rb2o_filter_table.restype = None
    t = np.zeros(256, np.float32)
    L.rb2o_filter_table(FILTER_KINDS[kind], xwidth, ywidth, alpha, _p(t))
    return t.reshape(16, 16)


def film(kind: str, xwidth: float, ywidth: float, alpha: float, width: int, height: int, spp: int, xy, L4):
    """Filtered reconstruction (rb2o_film): xy (spp*w*h, 2), L4 (spp*w*h, 4)
    sample-major; returns (h*w, 3) float32."""
    Lb = orc_lib()
    Lb.rb2o_film.argtypes = [C.c_uint32, C.c_float, C.c_float, C.c_float, C.c_uint32, C.c_uint32, C.c_uint32,
                             C.c_void_p, C.c_void_p, C.c_void_p]
    Lb.rb2o_film.restype = None
    xy = np.ascontiguousarray(xy, np.float32)
    L4 = np.ascontiguousarray(L4, np.float32)
    out = np.zeros((width * height, 3), np.float32)
    Lb.rb2o_film(FILTER_KINDS[kind], xwidth, ywidth, alpha, width, height, spp, _p(xy), _p(L4), _p(out))
    return out


def trace(nodes, woop, triidx, rays, any_hit=False, mask=None, counts=False, nthreads=0):
    """CPU restatement of the reference traversal.  Returns a structured hit
    array (prim, t, u, v) and, with counts=True, per-ray visit counts."""
    nodes = np.ascontiguousarray(nodes, np.uint32)
    woop = np.ascontiguousarray(woop, np.uint32)
    triidx = np.ascontiguousarray(triidx, np.uint32)
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    n = rays.shape[0]
    hits = np.empty(n, HIT_DTYPE)
    cnt = np.empty(n, COUNT_DTYPE) if counts else None
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    orc_lib().rb2o_trace(_p(nodes), _p(woop), _p(triidx), _p(rays), n, 1 if any_hit else 0, _p(m), _p(hits),
                         _p(cnt), int(nthreads))
    return (hits, cnt) if counts else hits


def woop_test(woop_row3, ray8, tmax):
    w = np.ascontiguousarray(woop_row3, np.uint32).reshape(12)
    r = np.ascontiguousarray(ray8, np.float32).reshape(8)
    tuv = np.zeros(3, np.float32)
    ok = orc_lib().rb2o_woop_test(_p(w), _p(r), float(tmax), _p(tuv))
    return bool(ok), tuv


def bruteforce(woop, triidx, rays, nthreads=0):
    woop = np.ascontiguousarray(woop, np.uint32)
    triidx = np.ascontiguousarray(triidx, np.uint32)
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    hits = np.empty(rays.shape[0], HIT_DTYPE)
    orc_lib().rb2o_bruteforce(_p(woop), _p(triidx), woop.reshape(-1, 4).shape[0], _p(rays), rays.shape[0],
                              _p(hits), int(nthreads))
    return hits


def tie_count(woop, triidx, rays, hits, nodes=None, nthreads=0) -> np.ndarray:
    """Per ray, how many distinct triangles accept it at exactly its
    closest-hit t (hits from `trace`): >= 2 marks a tie at a shared edge or
    vertex.  Without `nodes` every Woop slot is tested (exact, for small
    scenes); with the node buffer the BVH is walked with a slack around t
    (for statistics on large scenes)."""
    woop = np.ascontiguousarray(woop, np.uint32)
    triidx = np.ascontiguousarray(triidx, np.uint32)
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    hits = np.ascontiguousarray(hits, HIT_DTYPE)
    out = np.zeros(rays.shape[0], np.uint32)
    if nodes is None:
        orc_lib().rb2o_tie_count_brute(_p(woop), _p(triidx), woop.reshape(-1, 4).shape[0], _p(rays), rays.shape[0],
                                       _p(hits), _p(out), int(nthreads))
    else:
        nodes = np.ascontiguousarray(nodes, np.uint32)
        orc_lib().rb2o_tie_count(_p(nodes), _p(woop), _p(triidx), _p(rays), rays.shape[0], _p(hits), _p(out),
                                 int(nthreads))
    return out


def gen_heightfield(seed: int, grid_n: int, amplitude: float = 0.2, n_boxes: int = 64, box_min: float = 0.02,
                    box_max: float = 0.1):
    """The synthetic heightfield scene (oracle copy of the product generator):
    (vertices (nv, 3) float32, indices (nt, 3) uint32)."""
    nv, nt = C.c_uint32(), C.c_uint32()
    if orc_lib().rb2o_gen_heightfield_counts(grid_n, n_boxes, C.byref(nv), C.byref(nt)):
        raise ValueError("bad heightfield size")
    v = np.empty((nv.value, 3), np.float32)
    i = np.empty((nt.value, 3), np.uint32)
    if orc_lib().rb2o_gen_heightfield(seed, grid_n, amplitude, n_boxes, box_min, box_max, _p(v), _p(i)):
        raise RuntimeError("heightfield generation failed")
    return v, i


def gen_heightfield_for_triangles(seed: int, n_tris: int, n_boxes: int = 64):
    """Heightfield with a grid sized to about n_tris triangles (grid n =
    round(sqrt((T - 12 boxes) / 2)), the batching workload's rule)."""
    n = max(1, int(round(np.sqrt(max(2, n_tris - 12 * n_boxes) / 2.0))))
    return gen_heightfield(seed, n, n_boxes=n_boxes)


def gen_surface_rays(vertices, indices, seed: int, n: int, offset_scale: float = 1e-4,
                     anyhit_fraction: float = 0.5):
    """Incoherent diffuse-bounce rays from the scene's surfaces (oracle copy
    of the product generator): (rays (n, 8) float32, flags (n,) uint8)."""
    v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
    i = np.ascontiguousarray(indices, np.uint32).reshape(-1, 3)
    rays = np.empty((n, 8), np.float32)
    flags = np.empty((n,), np.uint8)
    if orc_lib().rb2o_gen_surface_rays(_p(v), v.shape[0], _p(i), i.shape[0], seed, n, offset_scale,
                                       anyhit_fraction, _p(rays), _p(flags)):
        raise ValueError("bad ray-generation arguments")
    return rays, flags


def ao_ref_dir(normal, u1, u2):
    """The reference's AO direction formula (oracle restatement, double);
    None where the reference's direction is NaN."""
    L = orc_lib()
    L.rb2o_ao_ref_dir.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_void_p]
    L.rb2o_ao_ref_dir.restype = C.c_int
    n = np.ascontiguousarray(normal, np.float64)
    out = np.zeros(3, np.float64)
    return out if L.rb2o_ao_ref_dir(_p(n), float(u1), float(u2), _p(out)) else None


def light_le_ref(light_normal, area, u3, u4):
    """DiffuseAreaLight::Le's direction and Le / pdf factor (oracle restatement)."""
    L = orc_lib()
    L.rb2o_light_le_ref.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_void_p,
                                    C.POINTER(C.c_double)]
    L.rb2o_light_le_ref.restype = None
    n = np.ascontiguousarray(light_normal, np.float64)
    d = np.zeros(3, np.float64)
    k = C.c_double()
    L.rb2o_light_le_ref(_p(n), float(area), float(u3), float(u4), _p(d), C.byref(k))
    return d, k.value


def ref_ao_direction(normal, u1, u2):
    """The reference's compiled cosine_sample_hemisphere_normal (float)."""
    L = ref_lib()
    L.rb2ref_ao_direction.argtypes = [C.c_float, C.c_float, C.c_void_p, C.c_void_p]
    L.rb2ref_ao_direction.restype = C.c_int
    n = np.ascontiguousarray(normal, np.float32)
    out = np.zeros(3, np.float32)
    L.rb2ref_ao_direction(float(u1), float(u2), _p(n), _p(out))
    return out


def ref_light_le(v0, v1, v2, emit, u5):
    """The reference's compiled DiffuseAreaLight::Le: (point, direction, pdf, L)."""
    L = ref_lib()
    L.rb2ref_light_le.argtypes = [C.c_void_p] * 9
    L.rb2ref_light_le.restype = C.c_int
    a = [np.ascontiguousarray(x, np.float32) for x in (v0, v1, v2, emit, u5)]
    pt, d, pdf, Lo = np.zeros(3, np.float32), np.zeros(3, np.float32), np.zeros(1, np.float32), np.zeros(3, np.float32)
    L.rb2ref_light_le(*[_p(x) for x in a], _p(pt), _p(d), _p(pdf), _p(Lo))
    return pt, d, float(pdf[0]), Lo


def woop_slots_of(woop, triidx):
    """Map from triangle id to its first Woop slot (for tie checks)."""
    w = np.asarray(woop, np.uint32).reshape(-1, 4)
    slots = {}
    s = 0
    n = w.shape[0]
    while s < n:
        if w[s, 0] == 0x80000000:
            s += 1
            continue
        slots.setdefault(int(triidx[s]), s)
        s += 3
    return slots


def is_tie(woop, triidx, slots, ray8, prim_a, prim_b) -> bool:
    """True when both triangles accept the ray at the same t (an edge/vertex tie)."""
    w = np.asarray(woop, np.uint32).reshape(-1, 4)
    if prim_a < 0 or prim_b < 0:
        return False
    sa, sb = slots.get(int(prim_a)), slots.get(int(prim_b))
    if sa is None or sb is None:
        return False
    big = np.float32(3.4028235e38)
    oka, tuva = woop_test(w[sa:sa + 3], ray8, big)
    okb, tuvb = woop_test(w[sb:sb + 3], ray8, big)
    return oka and okb and tuva[0] == tuvb[0]


# ---------------------------------------------------------------- shading references
class _Scene(C.Structure):
    _fields_ = [("verts", C.c_void_p), ("tris", C.c_void_p), ("tri_mat", C.c_void_p), ("albedo", C.c_void_p),
                ("emission", C.c_void_p), ("lights", C.c_void_p), ("n_lights", C.c_uint32),
                ("materials", C.c_void_p)]


# rb2o_layer / rb2o_material (the product's rb2_bsdf_layer / rb2_material_desc layout).
LAYER_DTYPE = np.dtype([("type", np.uint32), ("fresnel", np.uint32), ("color", np.float32, 3),
                        ("sigma_deg", np.float32), ("etai", np.float32), ("etat", np.float32),
                        ("exponent", np.float32), ("eta", np.float32, 3), ("k", np.float32, 3)])
MATERIAL_DTYPE = np.dtype([("n_layers", np.uint32), ("reserved", np.uint32), ("layer", LAYER_DTYPE, 4)])
assert LAYER_DTYPE.itemsize == 60 and MATERIAL_DTYPE.itemsize == 248


def materials_array(descs) -> np.ndarray:
    """Material descriptions as an rb2o_material array: `descs` is a ctypes
    rb2_material_desc array (same bytes) or a structured numpy array."""
    if isinstance(descs, np.ndarray):
        return np.ascontiguousarray(descs, MATERIAL_DTYPE)
    return np.frombuffer(bytes(descs), MATERIAL_DTYPE).copy()


def material_query(material, sample: bool, q) -> np.ndarray:
    """FP64 material functions (rb2o_material_query) for one material over
    queries q (n, 9); returns (n, 4) f/pdf or (n, 8) wi/f/pdf/specular."""
    m = materials_array(material).reshape(-1)[:1]
    q = np.ascontiguousarray(q, np.float64).reshape(-1, 9)
    L = orc_lib()
    L.rb2o_material_query.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    L.rb2o_material_query.restype = None
    w = 8 if sample else 4
    out = np.zeros((q.shape[0], w), np.float64)
    for i in range(q.shape[0]):
        L.rb2o_material_query(_p(m), 1 if sample else 0, _p(q[i]), out[i].ctypes.data)
    return out


def ref_material(material, sample: bool, q) -> np.ndarray:
    """The reference's material_f / material_pdf / material_sample_f (compiled
    from core/reflection.cu and core/material.cu) on the same queries."""
    m = materials_array(material).reshape(-1)[0]
    layers = np.ascontiguousarray(m["layer"][: int(m["n_layers"])])
    q = np.ascontiguousarray(q, np.float32).reshape(-1, 9)
    L = ref_lib()
    L.rb2ref_material.argtypes = [C.c_void_p, C.c_uint32, C.c_int, C.c_void_p, C.c_void_p]
    L.rb2ref_material.restype = C.c_int
    w = 8 if sample else 4
    out = np.zeros((q.shape[0], w), np.float32)
    for i in range(q.shape[0]):
        rc = L.rb2ref_material(_p(layers), int(m["n_layers"]), 1 if sample else 0, _p(q[i]), out[i].ctypes.data)
        if rc != 0:
            raise RuntimeError("reference material query failed")
    return out


class _Bvh(C.Structure):
    _fields_ = [("nodes", C.c_void_p), ("woop", C.c_void_p), ("triidx", C.c_void_p)]


def _scene_struct(vertices, indices, tri_mat, albedo, emission, lights, materials=None):
    keep = [np.ascontiguousarray(vertices, np.float32), np.ascontiguousarray(indices, np.uint32),
            np.ascontiguousarray(tri_mat, np.uint32), np.ascontiguousarray(albedo, np.float32),
            np.ascontiguousarray(emission, np.float32), np.ascontiguousarray(lights, np.uint32)]
    mats = None if materials is None else materials_array(materials)
    keep.append(mats)
    s = _Scene(*[_p(k) for k in keep[:6]], keep[5].shape[0], _p(mats))
    return s, keep


def _bvh_struct(nodes, woop, triidx):
    keep = [np.ascontiguousarray(nodes, np.uint32), np.ascontiguousarray(woop, np.uint32),
            np.ascontiguousarray(triidx, np.uint32)]
    return _Bvh(*[_p(k) for k in keep]), keep


def ao(bvh_buffers, vertices, indices, prim_rays, samples, radius, seed=1, nthreads=0, compat=0):
    """FP64 ambient occlusion per primary ray (see rb2_oracle.h); compat=1:
    the reference's AO direction formula."""
    L = orc_lib()
    L.rb2o_ao.argtypes = [C.POINTER(_Bvh), C.POINTER(_Scene), C.c_void_p, C.c_uint32, C.c_uint32, C.c_float,
                          C.c_uint64, C.c_uint32, C.c_void_p, C.c_int]
    L.rb2o_ao.restype = None
    n_tri = np.asarray(indices).reshape(-1, 3).shape[0]
    s, ks = _scene_struct(vertices, indices, np.zeros(n_tri, np.uint32), np.zeros((1, 3), np.float32),
                          np.zeros((1, 3), np.float32), np.zeros(1, np.uint32))
    b, kb = _bvh_struct(*bvh_buffers)
    r = np.ascontiguousarray(prim_rays, np.float32).reshape(-1, 8)
    out = np.empty(r.shape[0], np.float64)
    L.rb2o_ao(C.byref(b), C.byref(s), _p(r), r.shape[0], samples, radius, seed, compat, _p(out), nthreads)
    return out


def pt(bvh_buffers, vertices, indices, tri_mat, albedo, emission, lights, rays, max_depth, rr_start, rr_prob,
       seed=1, nthreads=0, materials=None, compat=0):
    """One FP64 path-traced sample per camera ray; returns (n, 3) radiance.
    `materials` (optional): layered material descriptions per material.
    compat: 2 = the reference's roulette divisor, 4 = its NEE re-seeding."""
    L = orc_lib()
    L.rb2o_pt.argtypes = [C.POINTER(_Bvh), C.POINTER(_Scene), C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
                          C.c_float, C.c_uint64, C.c_uint32, C.c_void_p, C.c_int]
    L.rb2o_pt.restype = None
    s, ks = _scene_struct(vertices, indices, tri_mat, albedo, emission, lights, materials)
    b, kb = _bvh_struct(*bvh_buffers)
    r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    out = np.empty((r.shape[0], 3), np.float64)
    L.rb2o_pt(C.byref(b), C.byref(s), _p(r), r.shape[0], max_depth, rr_start, rr_prob, seed, compat, _p(out),
              nthreads)
    return out


def bdpt(bvh_buffers, vertices, indices, tri_mat, albedo, emission, lights, cam_rays, n_cam, n_iter, n_light_paths,
         K, C, rr_start, rr_prob, seed=1, nthreads=0, materials=None):
    """FP64 BDPT-LVC mean radiance per camera pixel over n_iter iterations.

    `materials` (optional): layered material descriptions per material,
    mirror and glass layers included."""
    L = orc_lib()
    L.rb2o_bdpt.argtypes = [C_.POINTER(_Bvh), C_.POINTER(_Scene), C_.c_void_p, C_.c_uint32, C_.c_uint32, C_.c_uint32,
                            C_.c_uint32, C_.c_uint32, C_.c_uint32, C_.c_float, C_.c_uint64, C_.c_void_p, C_.c_int]
    L.rb2o_bdpt.restype = None
    s, ks = _scene_struct(vertices, indices, tri_mat, albedo, emission, lights, materials)
    b, kb = _bvh_struct(*bvh_buffers)
    r = np.ascontiguousarray(cam_rays, np.float32).reshape(-1, 8)
    assert r.shape[0] == n_cam * n_iter
    out = np.empty((n_cam, 3), np.float64)
    L.rb2o_bdpt(C_.byref(b), C_.byref(s), _p(r), n_cam, n_iter, n_light_paths, K, C, rr_start, rr_prob, seed, _p(out),
                nthreads)
    return out


C_ = C


class _BdptRefParams(C.Structure):
    _fields_ = [("n_prep", C.c_uint32), ("n_light_paths", C.c_uint32), ("light_max_depth", C.c_uint32),
                ("cam_max_depth", C.c_uint32), ("cam_rrstart", C.c_uint32), ("connections", C.c_uint32),
                ("cam_rrprob", C.c_float)]


def bdpt_ref(bvh_buffers, vertices, indices, tri_mat, albedo, emission, lights, cam_rays, n_cam, n_iter,
             n_prep, n_light_paths, light_max_depth, cam_max_depth, cam_rrstart, cam_rrprob, connections, seed=1,
             nthreads=0, materials=None):
    """FP64 restatement of the reference's own BDPT estimator
    (integrators/integrator_bdpt_lvc_sk.cu; see rb2_oracle.h): mean radiance
    per camera pixel over n_iter iterations (cam_rays iteration-major)."""
    L = orc_lib()
    L.rb2o_bdpt_ref.argtypes = [C.POINTER(_Bvh), C.POINTER(_Scene), C.c_void_p, C.c_uint32, C.c_uint32,
                                C.POINTER(_BdptRefParams), C.c_uint64, C.c_void_p, C.c_int]
    L.rb2o_bdpt_ref.restype = None
    s, ks = _scene_struct(vertices, indices, tri_mat, albedo, emission, lights, materials)
    b, kb = _bvh_struct(*bvh_buffers)
    r = np.ascontiguousarray(cam_rays, np.float32).reshape(-1, 8)
    assert r.shape[0] == n_cam * n_iter
    p = _BdptRefParams(n_prep, n_light_paths, light_max_depth, cam_max_depth, cam_rrstart, connections, cam_rrprob)
    out = np.empty((n_cam, 3), np.float64)
    L.rb2o_bdpt_ref(C.byref(b), C.byref(s), _p(r), n_cam, n_iter, C.byref(p), seed, _p(out), nthreads)
    return out


# ---- ray casting ---------------------------------------------------------------------
# kernel_ray_cast_update's colour table (integrators/integrator_raycast.cu:49-63).
RAYCAST_PALETTE = np.array([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0], [0.0, 1.0, 1.0], [1.0, 0.0, 1.0],
                            [1.0, 1.0, 0.0], [0.1, 0.1, 0.1], [0.5, 0.5, 0.5], [1.0, 1.0, 1.0], [0.0, 0.25, 0.5],
                            [1.0, 0.5, 0.0], [0.5, 0.25, 0.0], [0.2, 0.9, 1.0], [0.7, 0.3, 0.1],
                            [0.34, 0.89, 0.45]], np.float32)
_LAYER_OREN_NAYAR = 1


def raycast_shade(prim, mode, vertices, indices, tri_mat, albedo, emission, materials=None):
    """Colour per camera sample of the reference's ray-cast integrator
    (kernel_ray_cast_update, integrators/integrator_raycast.cu:37-131) from
    closest-hit primitive ids (-1 = miss), float32 (n, 3); misses are black:

    mode 0 (:65-71): the palette at prim mod 15;
    mode 1 (:72-109): the first layer's colour of the hit material (the
        emission of an emitter; black for Oren-Nayar, which has no branch
        there), with `materials` a material_descs array or None (one
        Lambertian layer = albedo per material);
    mode 2 (:110-116): the shading normal, here the unflipped geometric
        normal normalize(cross(v1 - v0, v2 - v0)) (float64, rounded);
    mode 3 (:117-120): black (the branch is empty);
    mode 4 (:121-124): one on a hit."""
    prim = np.asarray(prim).astype(np.int64).reshape(-1)
    hit = prim >= 0
    out = np.zeros((prim.size, 3), np.float32)
    p = prim[hit]
    if mode == 0:
        out[hit] = RAYCAST_PALETTE[p % 15]
    elif mode == 1:
        m = np.asarray(tri_mat, np.int64)[p]
        em = np.asarray(emission, np.float32).reshape(-1, 3)
        col = np.asarray(albedo, np.float32).reshape(-1, 3).copy()
        if materials is not None:
            arr = materials_array(materials)
            for k in range(arr.shape[0]):
                lay = arr[k]["layer"][0]
                if arr[k]["n_layers"] >= 1:
                    col[k] = 0.0 if lay["type"] == _LAYER_OREN_NAYAR else lay["color"]
        emitter = (em > 0).any(axis=1)
        col[emitter] = em[emitter]
        out[hit] = col[m]
    elif mode == 2:
        v = np.asarray(vertices, np.float64).reshape(-1, 3)
        t = np.asarray(indices, np.int64).reshape(-1, 3)[p]
        n = np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]])
        out[hit] = (n / np.linalg.norm(n, axis=1, keepdims=True)).astype(np.float32)
    elif mode == 4:
        out[hit] = 1.0
    return out


def _splitmix64(z):
    z = (z + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def keyed_u01_f32(seed, key, dim):
    """The integrators' keyed draw in [0, 1) as float32 (24 bits), restated so
    that tests can rebuild the device's sample positions: splitmix64 of
    (key * 0x100000001B3 + dim), xor seed, splitmix64 again, then the PCG32
    xorshift-and-rotate output permutation; the top 24 of its 32 bits give the
    value.  `key` is an integer array."""
    with np.errstate(over="ignore"):
        key = np.asarray(key, np.uint64)
        s = _splitmix64(np.uint64(seed) ^ _splitmix64(key * np.uint64(0x100000001B3) + np.uint64(dim)))
        xs = (((s >> np.uint64(18)) ^ s) >> np.uint64(27)) & np.uint64(0xFFFFFFFF)
        rot = s >> np.uint64(59)
        r = ((xs >> rot) | (xs << ((np.uint64(32) - rot) & np.uint64(31)))) & np.uint64(0xFFFFFFFF)
    return (r >> np.uint64(8)).astype(np.float32) * np.float32(1.0 / 16777216.0)


def jittered_raster(width, height, spp, seed, sample0=0):
    """Raster positions of the integrators' camera samples, sample-major
    (index = s * pixels + pixel): x = pixel % width + u(key, 0), y = pixel /
    width + u(key, 1), key = (sample0 + s) * pixels + pixel, float32 sums."""
    npix = width * height
    pix = np.tile(np.arange(npix, dtype=np.uint64), spp)
    s = np.repeat(np.arange(spp, dtype=np.uint64), npix) + np.uint64(sample0)
    key = s * np.uint64(npix) + pix
    jx, jy = keyed_u01_f32(seed, key, 0), keyed_u01_f32(seed, key, 1)
    x = (pix % np.uint64(width)).astype(np.float32) + jx
    y = (pix // np.uint64(width)).astype(np.float32) + jy
    return np.stack([x, y], 1)
