"""The bench's multi-GPU arithmetic (replicas: each rank runs the whole workload) with two gloo
ranks on the CPU: the job time is the slowest rank's, the value sums the replicas."""
import os
import sys
from pathlib import Path

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = [12.5, 17.25][rank]
        ms = bench.rank_max(local_ms, dist, "cpu")
        q.put((rank, ms, bench.job_value(world, 1000, 3, 10, ms)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_max_and_value():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in ps)
    res = sorted(q.get(timeout=5) for _ in range(2))
    for rank, ms, val in res:
        assert ms == 17.25                                   # slowest rank on every rank
        assert val == pytest.approx(2 * 1000 * 3 * 10 / 17.25e-3)


def test_single_process_passthrough():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.rank_max(3.0, None, "cpu") == 3.0
