"""Multi-GPU runs are independent replicas (one process per GPU): the host
logic of the N > 1 path -- distinct replica seeds, max-over-ranks timing,
whole-job throughput -- checked with world_size 2 over gloo on CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from mainline_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        local = [10.0 + rank, 5.0 - rank, 7.0 * (rank + 1)]
        out[rank] = (replicas.max_over_ranks(local, "cpu"), replicas.replica_seed(100, rank))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_time():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    (m0, s0), (m1, s1) = out[0], out[1]
    assert m0 == m1 == [11.0, 5.0, 14.0]
    assert s0 != s1


def test_single_rank_and_aggregate_rate():
    assert replicas.max_over_ranks([1.5, 2.0], "cpu") == [1.5, 2.0]
    # 4096 walkers x 100 steps on each of 8 replicas, slowest 1000 ms
    assert replicas.aggregate_rate(4096 * 100, 8, 1000.0) == pytest.approx(3276800.0)
