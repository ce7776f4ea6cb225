"""The multi-rank bench logic on CPU with two gloo ranks: every rank reports the slowest
rank's step time (max over ranks), and the job value is the aggregate of the replicas."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist)
        e2e = bench.max_over_ranks(3.0 - rank, dist)
        q.put((rank, ms, e2e, bench.aggregate_rate(world, 1024, ms)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    for rank, ms, e2e, value in res:
        assert ms == 15.0 and e2e == 3.0
        assert value == pytest.approx(2 * 1024 / 0.015)


def test_single_rank_passthrough():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(7.5) == 7.5
    assert bench.aggregate_rate(1, 100, 50.0) == pytest.approx(2000.0)
