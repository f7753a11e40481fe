"""The multi-process path of bench.py (one process per GPU, replicas) on the
CPU: two gloo ranks on 127.0.0.1 run the same barrier and max-over-ranks
aggregation as the NCCL ranks do, and the whole-job value follows from the
slowest rank."""
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

    from cudaplasticity_b200.ranks import max_over_ranks, replica_throughput

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        seconds = [1.5, 2.5][rank]  # this rank's timed region
        total = max_over_ranks(seconds, dist)
        out[rank] = (total, replica_throughput(world, 5, total))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_rank():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0] == res[1] == (2.5, 2 * 5 / 2.5)


def test_single_process_is_identity():
    from cudaplasticity_b200.ranks import max_over_ranks, replica_throughput

    assert max_over_ranks(3.0) == 3.0
    assert replica_throughput(1, 4, 2.0) == pytest.approx(2.0)
