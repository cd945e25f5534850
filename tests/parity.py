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
