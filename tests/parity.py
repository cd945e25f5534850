"""Shared comparison helpers for the parity tests."""
from __future__ import annotations

import numpy as np

GOLDEN = None


def golden():
    global GOLDEN
    if GOLDEN is None:
        from pathlib import Path
        GOLDEN = dict(np.load(Path(__file__).resolve().parent / "golden" / "golden_small.npz"))
    return GOLDEN


def split_hits(h):
    """(n,4) int32 device hit records -> prim, t, u, v."""
    h = np.asarray(h)
    f = h.view(np.float32)
    return h[:, 0], f[:, 1], f[:, 2], f[:, 3]


def compare_closest(orc, gpu_hits, ref_hits, woop, triidx, rays):
    """Closest-hit parity: prim, t, u and v must be bit-identical to the oracle
    except at ties (two triangles accepting the ray at the same t).  Returns
    (n_ties, n_bad, first_bad_index)."""
    gp, gt, gu, gv = split_hits(gpu_hits)
    same = (gp == ref_hits["prim"])
    bits_ok = same & (gt.view(np.uint32) == ref_hits["t"].view(np.uint32)) & \
        (gu.view(np.uint32) == ref_hits["u"].view(np.uint32)) & (gv.view(np.uint32) == ref_hits["v"].view(np.uint32))
    bad_idx = np.nonzero(~bits_ok)[0]
    ties = 0
    bad = []
    slots = orc.woop_slots_of(woop, triidx) if bad_idx.size else {}
    for k in bad_idx:
        if gp[k] != ref_hits["prim"][k] and gt[k] == ref_hits["t"][k] and \
                orc.is_tie(woop, triidx, slots, rays[k], gp[k], ref_hits["prim"][k]):
            ties += 1
        else:
            bad.append(int(k))
    return ties, len(bad), (bad[0] if bad else -1)


def compare_any(gpu_hits, ref_hits):
    """Any-hit parity: the occlusion decision must match exactly."""
    gp = np.asarray(gpu_hits)[:, 0]
    return int(((gp >= 0) != (ref_hits["prim"] >= 0)).sum())


def compare_closest_wide(orc, gpu_hits, ref_hits, woop, triidx, rays):
    """Closest-hit parity for the 4-wide and compressed 8-wide layouts, which
    test the same triangles in another order through boxes that contain the
    binary boxes.  A mismatch is allowed when it is
      * a confirmed tie (both triangles accept the ray at the same t), or
      * a reference-culled hit: the ray has a direction component exactly 0
        and runs exactly in a binary box's boundary plane, where the
        reference's slab test (zero replaced by +-2^-80) culls that box; the
        wide layout then reports the true nearest hit, so its t is smaller
        than the oracle's and equals the exhaustive search's.
    Returns (n_ties, n_reference_culled, n_bad, first_bad_index)."""
    gp, gt, gu, gv = split_hits(gpu_hits)
    same = (gp == ref_hits["prim"])
    bits_ok = same & (gt.view(np.uint32) == ref_hits["t"].view(np.uint32)) & \
        (gu.view(np.uint32) == ref_hits["u"].view(np.uint32)) & (gv.view(np.uint32) == ref_hits["v"].view(np.uint32))
    bad_idx = np.nonzero(~bits_ok)[0]
    ties = culled = 0
    bad = []
    if bad_idx.size:
        slots = orc.woop_slots_of(woop, triidx)
        bf = orc.bruteforce(woop, triidx, rays[bad_idx])
    for j, k in enumerate(bad_idx):
        axis_parallel = bool((rays[k, 4:7] == 0.0).any())
        if gp[k] != ref_hits["prim"][k] and gt[k] == ref_hits["t"][k] and \
                orc.is_tie(woop, triidx, slots, rays[k], gp[k], ref_hits["prim"][k]):
            ties += 1
        elif axis_parallel and gt[k] < ref_hits["t"][k] and gt[k] == bf["t"][j] and \
                (gp[k] == bf["prim"][j] or orc.is_tie(woop, triidx, slots, rays[k], gp[k], bf["prim"][j])):
            culled += 1
        else:
            bad.append(int(k))
    return ties, culled, len(bad), (bad[0] if bad else -1)
