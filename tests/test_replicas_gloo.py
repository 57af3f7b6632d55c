"""The N > 1 form of bench.py: N independent replicas, timed as the
slowest rank (max over ranks) and reported per unit of whole-job work.  Two
gloo ranks on CPU run the same aggregation code as the NCCL ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = 10.0 * (rank + 1)  # rank 1 is the slower replica
        total = bench.max_over_ranks(mine, world, device="cpu")
        out[rank] = (total,) + bench.replica_rates(total, 5, world)
    finally:
        dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        total, per_step, value = res[r]
        assert total == 20.0  # the slowest rank, on every rank
        assert per_step == pytest.approx(4.0) and value == pytest.approx(2.0)


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(7.5, 1) == 7.5
    assert bench.replica_rates(7.5, 3, 1) == (2.5, 2.5)
