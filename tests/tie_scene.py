"""Geometry and rays that produce exact ties for the tie-rule tests.

A flat 16 x 16 grid on y = 0 and floating axis-aligned boxes, every vertex
coordinate a multiple of 1/16, so each triangle's Woop rows are exact and
coplanar (or edge-sharing) triangles agree on t to the last bit.  Rays are
aimed, with dyadic directions and origins, at lattice vertices, edge and
diagonal midpoints, box edges and box corners; along such a ray every
operation of the Woop test is exact, so two or more triangles accept the ray
at the same t.  The reference resolves ties by its acceptance rule
`tmin < t < hitT` (accelerators/sbvh/cuda_tracer_functions.cu:188-208,
accelerators/sbvh/kepler_dynamic_fetch.h:264): the triangle tested first
keeps the hit."""
from __future__ import annotations

import numpy as np

N = 16
# (lo, hi) corners in grid units (1/16).
BOXES = [((2, 2, 2), (5, 5, 4)), ((9, 3, 8), (12, 6, 13)), ((4, 1, 10), (7, 2, 12))]
_FACES = [(0, 4, 6, 2), (1, 3, 7, 5), (0, 1, 5, 4), (2, 6, 7, 3), (0, 2, 3, 1), (4, 5, 7, 6)]


def tie_scene(rb):
    """The flat grid plus boxes as an rb2 Scene."""
    vs, ids = [], []
    for j in range(N + 1):
        for i in range(N + 1):
            vs.append((i / N, 0.0, j / N))
    for j in range(N):
        for i in range(N):
            v00 = j * (N + 1) + i
            v10, v01 = v00 + 1, v00 + N + 1
            v11 = v01 + 1
            ids += [(v00, v01, v11), (v00, v11, v10)]
    for lo, hi in BOXES:
        b = len(vs)
        for k in range(8):
            vs.append(tuple((hi[a] if (k >> a) & 1 else lo[a]) / N for a in range(3)))
        for a, c1, c2, d in _FACES:
            ids += [(b + a, b + c1, b + c2), (b + a, b + c2, b + d)]
    s = rb.Scene()
    s.vertices = np.asarray(vs, np.float32)
    s.indices = np.asarray(ids, np.uint32)
    s.material_ids = np.zeros((s.indices.shape[0],), np.uint32)
    return s


def _aim(targets, d, back=2.0):
    t = np.asarray(targets, np.float32).reshape(-1, 3)
    d = np.asarray(d, np.float32).reshape(-1, 3)
    d = np.broadcast_to(d, t.shape)
    r = np.zeros((t.shape[0], 8), np.float32)
    r[:, 0:3] = t - np.float32(back) * d
    r[:, 4:7] = d
    r[:, 7] = np.float32(3.4028235e38)
    return r


def tie_rays():
    """(rays (n, 8) float32, kind (n,) str): the tie-producing ray set."""
    g = np.arange(1, N, dtype=np.float32) / N
    h = (np.arange(0, N, dtype=np.float32) + 0.5) / N
    verts = [(x, 0.0, z) for x in g for z in g]
    edges = [(x, 0.0, z) for x in h for z in g] + [(x, 0.0, z) for x in g for z in h]
    diags = [(x, 0.0, z) for x in h for z in h]
    rays, kinds = [], []

    def add(kind, targets, dirs):
        for d in dirs:
            r = _aim(targets, d)
            rays.append(r)
            kinds.extend([kind] * r.shape[0])

    down = [(0.0, -1.0, 0.0)]
    oblique = [(0.25, -1.0, 0.125), (-0.5, -1.0, 0.25), (0.125, -0.5, -0.5)]
    grazing = [(1.0, -1.0 / 32, 0.0), (0.0, -1.0 / 32, -1.0), (-1.0, -1.0 / 64, 0.5)]
    add("vertex", verts, down + oblique + grazing)
    add("edge", edges, down + oblique + grazing)
    add("diagonal", diags, down + oblique + grazing)
    # Box edges and corners, hit from outside across the edge / corner.
    box_edge, box_corner = [], []
    for lo, hi in BOXES:
        lo = np.asarray(lo, np.float32) / N
        hi = np.asarray(hi, np.float32) / N
        mid = (lo + hi) / 2
        # top edges (shared by the top face and a side face)
        box_edge.append(((lo[0], hi[1], mid[2]), (0.5, -0.5, 0.0)))
        box_edge.append(((hi[0], hi[1], mid[2]), (-0.5, -0.5, 0.0)))
        box_edge.append(((mid[0], hi[1], lo[2]), (0.0, -0.5, 0.5)))
        box_edge.append(((mid[0], hi[1], hi[2]), (0.0, -0.5, -0.5)))
        # vertical edges (two side faces)
        box_edge.append(((lo[0], mid[1], lo[2]), (0.5, 0.0, 0.25)))
        box_edge.append(((hi[0], mid[1], hi[2]), (-0.25, 0.0, -0.5)))
        # face diagonals (the two triangles of one face)
        box_edge.append(((mid[0], hi[1], mid[2]), (0.0, -1.0, 0.0)))
        box_edge.append(((lo[0], mid[1], mid[2]), (1.0, 0.0, 0.0)))
        for cx in (lo[0], hi[0]):
            for cz in (lo[2], hi[2]):
                dx = 0.5 if cx == lo[0] else -0.5
                dz = 0.25 if cz == lo[2] else -0.25
                box_corner.append(((cx, hi[1], cz), (dx, -0.5, dz)))
    for kind, items in (("box_edge", box_edge), ("box_corner", box_corner)):
        for tgt, d in items:
            r = _aim([tgt], d)
            rays.append(r)
            kinds.append(kind)
    return np.concatenate(rays, 0), np.asarray(kinds)
