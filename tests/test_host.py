"""CPU tests of librb2's host side: C-ABI exports, error behaviour, builder
edge cases, layout validation and the BVH cache formats."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from parity import golden

ROOT = Path(__file__).resolve().parent.parent


def _declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(rb2_\w+)\s*\(", text, re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol(rb):
    names = _declared_functions()
    assert len(names) > 20
    out = subprocess.run(["nm", "-D", "--defined-only", str(ROOT / "renderbox2_b200/_lib/librb2.so")],
                         capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = sorted(n for n in names if n not in exported)
    assert not missing, f"declared but not exported: {missing}"
    L = rb.lib()
    for n in names:
        getattr(L, n)


def test_errors_are_status_codes(rb):
    L = rb.lib()
    h = C.c_void_p()
    rc = L.rb2_bvh_build(None, 0, None, 5, None, C.byref(h))
    assert rc == 1 and b"null" in L.rb2_last_error()
    rc = L.rb2_bvh_load(b"/nonexistent/file.bvh", C.byref(h))
    assert rc == 4
    v = np.zeros((3, 3), np.float32)
    i = np.array([[0, 1, 7]], np.uint32)
    rc = L.rb2_bvh_build(v.ctypes.data, 3, i.ctypes.data, 1, None, C.byref(h))
    assert rc == 1 and b"out of range" in L.rb2_last_error()


@pytest.mark.parametrize("ntri", [0, 1, 2, 5])
def test_build_tiny_inputs(rb, orc, ntri):
    rng = np.random.Generator(np.random.PCG64(ntri))
    v = rng.uniform(0, 1, size=(3 * ntri, 3)).astype(np.float32)
    i = np.arange(3 * ntri, dtype=np.uint32).reshape(-1, 3)
    b = rb.BVH(rb.Scene().add_mesh(v, i))
    st = b.stats()
    assert st["n_inner"] >= 1 and st["n_nodes_u4"] % 4 == 0
    rays = np.zeros((64, 8), np.float32)
    rays[:, 0:3] = rng.uniform(-1, 2, size=(64, 3))
    d = rng.normal(size=(64, 3))
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 7] = 1e30
    h = orc.trace(b.get_node_buffer(), b.get_tri_woop_buffer(), b.get_tri_index_buffer(), rays)
    bf = orc.bruteforce(b.get_tri_woop_buffer(), b.get_tri_index_buffer(), rays)
    assert np.array_equal(h["prim"], bf["prim"])


def test_degenerate_and_duplicate_triangles(rb, orc):
    s = rb.heightfield_scene(seed=5, grid_n=8, n_boxes=2)
    v = np.concatenate([s.vertices, np.array([[0.3, 0.5, 0.3], [0.3, 0.5, 0.3], [0.3, 0.5, 0.3]], np.float32)])
    n0 = s.vertices.shape[0]
    extra = np.array([[n0, n0 + 1, n0 + 2], [0, 1, 2]], np.uint32)  # a point triangle and a duplicate
    i = np.concatenate([s.indices, extra])
    b = rb.BVH(rb.Scene().add_mesh(v, i))
    tri = set(b.get_tri_index_buffer()[b.get_tri_woop_buffer()[:, 0] != 0x80000000].tolist())
    assert (i.shape[0] - 2) not in tri  # degenerate (point) triangle removed, as the reference does
    rays, _ = rb.surface_rays(s, seed=6, n=4000)
    h = orc.trace(b.get_node_buffer(), b.get_tri_woop_buffer(), b.get_tri_index_buffer(), rays)
    bf = orc.bruteforce(b.get_tri_woop_buffer(), b.get_tri_index_buffer(), rays)
    assert np.array_equal(h["t"].view(np.uint32), bf["t"].view(np.uint32))


def test_builder_deterministic_across_thread_counts(rb):
    s = rb.heightfield_scene(seed=8, grid_n=200, n_boxes=32)
    b1 = rb.BVH(s, params=rb.BuildParams(num_threads=1))
    b8 = rb.BVH(s, params=rb.BuildParams(num_threads=8))
    assert np.array_equal(b1.get_node_buffer(), b8.get_node_buffer())
    assert np.array_equal(b1.get_tri_woop_buffer(), b8.get_tri_woop_buffer())


def test_benchmark_build_costs_make_smaller_leaves_with_the_same_hits(rb, orc):
    """The benchmark workloads build with SAH triangle cost 2
    (configs.BUILD) instead of the reference's 1: leaves hold fewer triangle
    references, the tree stays valid, and the closest hit distance of every
    ray equals the exhaustive search's on both trees."""
    from renderbox2_b200.configs import BUILD
    s = rb.heightfield_for_triangles(seed=31, n_tris=20_000, n_boxes=16)
    ref = rb.BVH(s)
    gpu = rb.BVH(s, platform=rb.Platform(sah_node_cost=BUILD["sah_node_cost"],
                                          sah_triangle_cost=BUILD["sah_triangle_cost"]))
    assert BUILD["sah_triangle_cost"] > 1.0
    per_leaf = [b.stats()["n_tri_refs"] / b.stats()["n_leaves"] for b in (ref, gpu)]
    assert per_leaf[1] < per_leaf[0], per_leaf
    rays, _ = rb.surface_rays(s, seed=32, n=20_000)
    for b in (ref, gpu):
        h = orc.trace(b.get_node_buffer(), b.get_tri_woop_buffer(), b.get_tri_index_buffer(), rays)
        bf = orc.bruteforce(b.get_tri_woop_buffer(), b.get_tri_index_buffer(), rays)
        assert np.array_equal(h["t"].view(np.uint32), bf["t"].view(np.uint32))


def test_spatial_splits_duplicate_long_triangles(rb, orc):
    # Long thin diagonal triangles overlap heavily: the SBVH should split some.
    rng = np.random.Generator(np.random.PCG64(3))
    n = 400
    a = rng.uniform(0, 1, size=(n, 3)).astype(np.float32)
    b_ = (a + rng.normal(scale=0.5, size=(n, 3))).astype(np.float32)
    c = (a + rng.normal(scale=0.01, size=(n, 3))).astype(np.float32)
    v = np.stack([a, b_, c], 1).reshape(-1, 3)
    i = np.arange(3 * n, dtype=np.uint32).reshape(-1, 3)
    bvh = rb.BVH(rb.Scene().add_mesh(v, i))
    assert bvh.stats()["n_tri_refs"] > n
    rays = np.zeros((5000, 8), np.float32)
    rays[:, 0:3] = rng.uniform(-0.5, 1.5, size=(5000, 3))
    d = rng.normal(size=(5000, 3))
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 7] = 1e30
    h = orc.trace(bvh.get_node_buffer(), bvh.get_tri_woop_buffer(), bvh.get_tri_index_buffer(), rays)
    bf = orc.bruteforce(bvh.get_tri_woop_buffer(), bvh.get_tri_index_buffer(), rays)
    assert np.array_equal(h["t"].view(np.uint32), bf["t"].view(np.uint32))


def test_validation_rejects_corrupt_layouts(rb):
    g = golden()
    nodes, woop, tri = g["ref_nodes"].copy(), g["ref_woop"].copy(), g["ref_triidx"].copy()
    rb.BVH.from_buffers(nodes, woop, tri)  # valid
    bad = nodes.copy()
    bad[3, 0] = 4 * (nodes.shape[0] // 4 + 10)  # child index past the end
    with pytest.raises(rb.Rb2Error):
        rb.BVH.from_buffers(bad, woop, tri)
    cyc = nodes.copy()
    cyc[3, 0] = 0  # root as its own child
    with pytest.raises(rb.Rb2Error):
        rb.BVH.from_buffers(cyc, woop, tri)
    unterminated = woop.copy()
    unterminated[unterminated[:, 0] == 0x80000000] = 0
    with pytest.raises(rb.Rb2Error):
        rb.BVH.from_buffers(nodes, unterminated, tri)
    with pytest.raises(rb.Rb2Error):
        rb.BVH.from_buffers(nodes[:5], woop, tri)


def test_binary_cache_round_trip(rb, tmp_path):
    s = rb.heightfield_scene(seed=9, grid_n=24, n_boxes=4)
    b = rb.BVH(s)
    p = tmp_path / "a.rb2bvh"
    b.serialize(str(p))
    c = rb.BVH.load(str(p))
    assert np.array_equal(b.get_node_buffer(), c.get_node_buffer())
    assert np.array_equal(b.get_tri_woop_buffer(), c.get_tri_woop_buffer())
    assert np.array_equal(b.get_tri_index_buffer(), c.get_tri_index_buffer())
    assert c.stats()["sah"] == b.stats()["sah"]
    raw = bytearray(p.read_bytes())
    raw[-5] ^= 0xFF
    p.write_bytes(bytes(raw))
    with pytest.raises(rb.Rb2Error) as e:
        rb.BVH.load(str(p))
    assert e.value.code == 5
    p.write_bytes(bytes(raw[:100]))
    with pytest.raises(rb.Rb2Error):
        rb.BVH.load(str(p))


def test_reads_reference_text_cache(rb):
    """The reference's own serialize() output (fixture) loads into rb2."""
    g = golden()
    c = rb.BVH.load(str(ROOT / "tests/golden/ref_cache_small.txt"))
    assert np.array_equal(c.get_node_buffer(), g["ref_nodes"])
    assert np.array_equal(c.get_tri_woop_buffer(), g["ref_woop"])
    assert np.array_equal(c.get_tri_index_buffer(), g["ref_triidx"])


def test_reference_reads_rb2_text_cache(rb, orc, tmp_path):
    if not orc.have_ref():
        pytest.skip("reference sources not compiled here")
    s = rb.heightfield_scene(seed=10, grid_n=12, n_boxes=2)
    b = rb.BVH(s)
    p = tmp_path / "x.txt"
    b.serialize_text(str(p))
    r = orc.ref_load(str(p))
    assert np.array_equal(r["nodes"], b.get_node_buffer())
    assert np.array_equal(r["woop"], b.get_tri_woop_buffer())
    assert np.array_equal(r["triidx"], b.get_tri_index_buffer())


def test_generators_are_seeded(rb):
    a = rb.heightfield_scene(seed=3, grid_n=16, n_boxes=4)
    b = rb.heightfield_scene(seed=3, grid_n=16, n_boxes=4)
    c = rb.heightfield_scene(seed=4, grid_n=16, n_boxes=4)
    assert np.array_equal(a.vertices, b.vertices) and not np.array_equal(a.vertices, c.vertices)
    assert a.num_triangles == 2 * 16 * 16 + 12 * 4
    r1, f1 = rb.surface_rays(a, seed=1, n=1000)
    r2, f2 = rb.surface_rays(a, seed=1, n=1000)
    assert np.array_equal(r1, r2) and np.array_equal(f1, f2)
    assert 0.4 < f1.mean() < 0.6
    d = r1[:, 4:7]
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-5)
    room = rb.RoomScene(seed=2, n_boxes=3, n_spheres=5, sphere_subdiv=2, n_lights=2)
    assert room.num_lights == 4
    assert room.emission[room.material_ids[room.light_ids_to_primitive_ids]].min() == 10.0


def test_job_footprints_and_arrivals(rb):
    import ctypes as C_
    from renderbox2_b200.serve import Job, _lib, poisson_arrivals
    L = _lib()
    j = Job()
    j.kind, j.n_rays, j.mode = 0, 1000, 0
    assert L.rb2_job_footprint(C_.byref(j)) == 1000 * 48
    j.mode = 2
    assert L.rb2_job_footprint(C_.byref(j)) == 1000 * 33
    t = Job()
    t.kind, t.tile, t.spp = 1, 256, 4
    small = L.rb2_job_footprint(C_.byref(t))
    t.tile = 1024
    big = L.rb2_job_footprint(C_.byref(t))
    assert big > 10 * small > 0
    a = poisson_arrivals(5000, rate=100.0, seed=1)
    assert np.all(np.diff(a) > 0) and abs(5000 / a[-1] - 100.0) < 5.0


def _compile_cpp(src, out, extra=()):
    import shutil
    import subprocess
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    lib = root / "renderbox2_b200" / "_lib"
    cmd = ["g++", "-std=c++17", "-O1", f"-I{root / 'include'}", "-I/usr/local/cuda/include", str(src),
           f"-L{lib}", "-lrb2", f"-Wl,-rpath,{lib}", *extra, "-o", str(out)]
    subprocess.run(cmd, check=True, capture_output=True)


def _fnv(b: bytes) -> int:
    h = 1469598103934665603
    for x in b:
        h = ((h ^ x) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def test_cpp_compat_classes_build_and_cache(rb, tmp_path):
    """rb2.hpp's reference-named classes (Scene/Mesh/BVH/CudaBvh) from C++:
    the buffers equal a build of the same triangles through the Python layer,
    and serialize() -> CudaBvh(file, ok) round-trips."""
    import subprocess
    from pathlib import Path
    src = Path(__file__).resolve().parent / "cpp" / "compat_host.cpp"
    exe = tmp_path / "compat_host"
    _compile_cpp(src, exe)
    out = subprocess.run([str(exe), str(tmp_path / "c.bvh")], check=True, capture_output=True, text=True).stdout
    f = dict(zip(out.split()[0::2], out.split()[1::2]))
    assert f["roundtrip"] == "1" and f["threw"] == "1"
    assert int(f["tris"]) == 1154 and int(f["lights"]) == 2
    # The same triangles through the Python layer.
    g = 24
    xs = np.arange(g + 1)
    verts = []
    for z in range(g + 1):
        for x in range(g + 1):
            y = np.float32(0.05) * np.float32((x * 7 + z * 3) % 5) / np.float32(4.0)
            verts.append((np.float32(x) / np.float32(g), y, np.float32(z) / np.float32(g)))
    idx = []
    for z in range(g):
        for x in range(g):
            a = z * (g + 1) + x
            b, c = a + 1, a + g + 1
            idx += [(a, c, b), (b, c, c + 1)]
    base = len(verts)
    verts += [(0.4, 0.9, 0.4), (0.6, 0.9, 0.4), (0.4, 0.9, 0.6), (0.6, 0.9, 0.6)]
    idx += [(base, base + 2, base + 1), (base + 1, base + 2, base + 3)]
    del xs
    sc = rb.Scene()
    sc.add_mesh(np.asarray(verts, np.float32), np.asarray(idx, np.uint32))
    bvh = rb.BVH(sc)
    nodes, woop, _ = bvh.buffers_view()
    assert int(f["nodes"]) == nodes.shape[0] and int(f["woop"]) == woop.shape[0]
    assert int(f["hash"], 16) == _fnv(np.ascontiguousarray(nodes).tobytes())


@pytest.mark.parametrize("kind,alpha", [("box", 0.0), ("triangle", 0.0), ("gaussian", 2.0), ("gaussian", 0.5)])
def test_filter_table_equals_oracle(rb, orc, kind, alpha):
    from renderbox2_b200.render import Filter, filter_table
    for xw, yw in ((0.5, 0.5), (1.5, 2.0), (2.0, 2.0), (3.7, 1.0)):
        got = filter_table(Filter(kind, xw, yw, alpha))
        want = orc.filter_table(kind, xw, yw, alpha)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    if kind == "triangle":
        t = filter_table(Filter(kind, 2.0, 1.0))
        assert not np.allclose(t[0, :], t[0, 0])   # varies along x (the reference's table did not)


def test_filter_validation_and_pfm(rb, tmp_path):
    from renderbox2_b200.render import Filter, filter_table, write_pfm
    for bad in (Filter("box", 0.0, 1.0), Filter("box", 1.0, 17.0), Filter("gaussian", 1.0, 1.0, 0.0)):
        with pytest.raises(rb.Rb2Error):
            filter_table(bad)
    img = np.arange(5 * 3 * 3, dtype=np.float32).reshape(15, 3)
    path = tmp_path / "a.pfm"
    write_pfm(path, img, 5, 3)
    raw = path.read_bytes()
    head = b"PF\n5 3\n-1.0\n"
    assert raw.startswith(head)
    data = np.frombuffer(raw[len(head):], "<f4").reshape(3, 5, 3)
    assert np.array_equal(data[::-1].reshape(15, 3), img)    # bottom row first
    with pytest.raises(rb.Rb2Error):
        write_pfm(tmp_path / "missing_dir" / "b.pfm", img, 5, 3)
