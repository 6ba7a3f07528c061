"""The multi-GPU bench path on CPU: world-size-2 gloo ranks, each timing its
own replica; the job time is the slowest rank's and the throughput counts
every rank's evaluations."""
from __future__ import annotations

import os
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        secs = [2.0, 5.0][rank]  # rank 1 is the slow replica
        slowest = bench.max_over_ranks(secs, world, device="cpu")
        out.put((rank, slowest, bench.replica_throughput(world, 3, slowest)))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_report_the_slowest_replica():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [5.0, 5.0]
    assert res[0][2] == pytest.approx(2 * 3 / 5.0)


def test_single_rank_is_its_own_time():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(1.5, 1) == 1.5
    assert bench.replica_throughput(1, 2, 4.0) == 0.5
