"""The bench's parity gate on the CPU: bench.parity_check, fed records equal
to the oracle's, reports no mismatch; with a mistake planted in the oracle's
own results (a closest-hit distance one float step off, an any-hit decision
flipped) it counts exactly those rays as mismatches and names the first one.
The GPU records the bench compares in the same way come from the timed
launch; here the oracle stands in for them."""
import numpy as np


def _case(rb):
    sc = rb.heightfield_for_triangles(seed=31, n_tris=4000)
    bvh = rb.BVH(sc)
    rays, _ = rb.surface_rays(sc, seed=32, n=4096)
    return [dict(bvh=bvh, rays=rays, n_ch=2048)]


def _records(samples):
    got_ch = [s["ch"]["hits"].copy().view(np.int32).reshape(-1, 4) for s in samples]
    got_occ = [(s["ah"]["hits"]["prim"] >= 0).astype(np.uint8) for s in samples]
    return got_ch, got_occ


def test_parity_gate_passes_equal_records_and_counts_planted_mistakes(rb, orc):
    import bench
    scenes = _case(rb)
    samples = bench.oracle_sample(scenes, 512)
    got_ch, got_occ = _records(samples)
    r = bench.parity_check(scenes, samples, got_ch, got_occ)
    assert r["rays"] == 1024 and r["mismatches"] == 0 and "first_mismatch" not in r

    hits = samples[0]["ch"]["hits"]
    k = int(np.nonzero(hits["prim"] >= 0)[0][3])
    hits["t"][k] = np.nextafter(hits["t"][k], np.float32(np.inf))  # the oracle's t, one step farther
    ah = samples[0]["ah"]["hits"]
    j = 7
    ah["prim"][j] = -1 if ah["prim"][j] >= 0 else 0  # the oracle's any-hit decision, flipped
    r = bench.parity_check(scenes, samples, got_ch, got_occ)
    assert r["mismatches"] == 2 and r["tie_divergent"] == 0
    assert r["first_mismatch"]["mode"] == "closest"
    assert r["first_mismatch"]["ray"] == int(samples[0]["ch"]["idx"][k])
