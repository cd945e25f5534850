"""The N > 1 host logic of bench.py on CPU: two gloo ranks (replicas, no
data-path collective).  Covers the barrier, the max-over-ranks time and the
whole-job rate (all ranks' units over the slowest rank's time), and that the
reference arm does no work on ranks other than 0."""
import json
import multiprocessing as mp
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import datetime

    import torch
    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        local_ms = 10.0 * (rank + 1)          # rank 1 is the slow one
        rate, ms = bench.whole_job_rate(1000.0, local_ms, world, torch.device("cpu"))
        mx = bench.max_over_ranks(float(rank) + 0.5, world, torch.device("cpu"))

        class A:
            scenes, rays_per_scene, ref_rays_per_scene, steps, warmup = 1, 64, 8, 1, 0
        ref = bench.run_reference(A, rank, world) if rank != 0 else None
        Path(out_dir, f"r{rank}.json").write_text(json.dumps({"rate": rate, "ms": ms, "max": mx, "ref": ref}))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_replica_rate(tmp_path):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("rank did not finish")
        assert p.exitcode == 0
    res = [json.loads((tmp_path / f"r{r}.json").read_text()) for r in range(2)]
    for r in res:
        assert r["ms"] == pytest.approx(20.0)               # slowest rank's time on every rank
        assert r["rate"] == pytest.approx(2 * 1000.0 / 0.020)  # both ranks' units / max time
        assert r["max"] == pytest.approx(1.5)
    assert res[1]["ref"] is None                            # reference arm: rank 1 does nothing
