"""The multi-rank bench path on the CPU: two gloo ranks, each timing its own
replica, agree on the slowest rank's time and on the whole-job value (the
path has no data-path collective: cones are independent, every rank solves a
replica)."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = 1.0 + rank  # rank 1 is the slower replica
        slowest = bench.max_over_ranks(mine, world, "cpu")
        out[rank] = (slowest, bench.replica_value(1000, 4, world, slowest))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_replica():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        got = dict(out)
    assert got[0] == got[1] == (2.0, 2 * 1000 * 4 / 2.0)


def test_one_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5
    assert bench.replica_value(10, 2, 1, 4.0) == pytest.approx(5.0)
