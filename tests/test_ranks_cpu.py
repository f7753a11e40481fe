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


# ---- instance sharding of the batched / served workloads (no GPU) ----

def test_partition_is_lpt_deterministic_and_covers_every_request():
    from cudaplasticity_b200.shard import partition

    parts = partition([5, 4, 3, 3, 3], 2)
    # 5 -> rank 0; 4 -> 1; 3 -> 1 (4 < 5); 3 -> 0 (5 < 7); 3 -> 1 (7 < 8)
    assert parts == [[0, 3], [1, 2, 4]]
    assert partition([5, 4, 3, 3, 3], 2) == parts
    costs = [float((7 * i) % 11 + 1) for i in range(40)]
    for world in (1, 2, 3, 8):
        ps = partition(costs, world)
        assert len(ps) == world
        assert sorted(i for p in ps for i in p) == list(range(40))
        assert all(p == sorted(p) for p in ps)
        loads = [sum(costs[i] for i in p) for p in ps]
        # LPT: no rank carries more than the mean plus the largest single cost
        assert max(loads) <= sum(costs) / world + max(costs)
    assert partition([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        partition([1.0], 0)


def test_request_cost_counts_increments():
    from cudaplasticity_b200.shard import request_cost

    assert request_cost(1000, 1) == 1000.0
    assert request_cost(1000, 5) == 5000.0
    assert request_cost(1000, 0) == 1000.0


class _FakeGather:
    """An all-gather over ranks whose records are given up front."""

    def __init__(self, parts):
        self.parts = parts

    def get_world_size(self):
        return len(self.parts)

    def all_gather_object(self, out, obj):
        for k, p in enumerate(self.parts):
            out[k] = p


def test_gather_rejects_a_request_solved_twice():
    from cudaplasticity_b200.shard import gather_records

    with pytest.raises(RuntimeError):
        gather_records({}, _FakeGather([{0: {"status": 0}}, {0: {"status": 0}}]))
    merged = gather_records({}, _FakeGather([{0: {"a": 1}}, {1: {"a": 2}}]))
    assert merged == {0: {"a": 1}, 1: {"a": 2}}


def _shard_rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from cudaplasticity_b200 import shard

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        n = 7
        costs = [float(i % 3 + 1) for i in range(n)]
        parts = shard.partition(costs, world)
        ticks = iter(range(1000))
        solved = []

        def build(i):
            return {"index": i, "cost": costs[i]}

        def submit(req):
            solved.append(req["index"])
            return req["index"]

        def wait(rid):
            return {"status": 0 if rid != 5 else 4, "latency": 0.1 * (rid + 1), "checksum": rid * 1.5,
                    "rank": rank}

        recs = shard.run_share(parts[rank], build, submit, wait, clock=lambda: float(next(ticks)))
        merged = shard.gather_records(recs, dist)
        summ = shard.summarize(merged, n, world)
        out[rank] = (sorted(solved), parts, sorted(merged), [merged[i]["rank"] for i in range(n)],
                     [merged[i]["checksum"] for i in range(n)], summ)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_the_requests_and_merge_the_records():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_shard_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    solved0, parts, keys0, owner, checks, summ0 = res[0]
    solved1, _, keys1, _, _, summ1 = res[1]
    # each rank solved exactly its share, the shares are disjoint and complete
    assert solved0 == parts[0] and solved1 == parts[1]
    assert sorted(solved0 + solved1) == list(range(7))
    # every rank holds the same merged records, with the right owners
    assert keys0 == keys1 == list(range(7))
    assert owner == [0 if i in parts[0] else 1 for i in range(7)]
    assert checks == [i * 1.5 for i in range(7)]
    assert summ0 == summ1
    assert summ0["statuses"] == [0, 4]
    assert summ0["requests"] == 7 and summ0["ranks"] == 2
    # the span is the slowest rank's: done_at counts clock ticks after the first submission
    longest = max(len(p) for p in parts)
    assert summ0["seconds"] == pytest.approx(float(longest))
    assert summ0["solves_per_s"] == pytest.approx(7 / float(longest))


def _bench_shard_rank(rank, world, port, fail_rank, out):
    """bench.py's sharded leg with a stand-in solve service (no GPU): the
    batch-stream meshes are built by the library's host code, the solves are
    faked; ``fail_rank``'s service fails to start."""
    import datetime

    import numpy as np
    import torch.distributed as dist

    import bench
    import cudaplasticity_b200 as cp

    class FakeInstance:
        def __init__(self, n):
            self.n = n

        def field(self, name):
            return np.full(2 * self.n, 0.5)

        def close(self):
            pass

    class FakeServer:
        def __init__(self, device=0, fp64_lanes=8):
            if rank == fail_rank:
                raise RuntimeError("service failed to start")
            self.meshes = []

        def submit(self, mesh, material, rp, mask, uv, **kw):
            self.meshes.append(len(mesh["node_xy"]))
            return len(self.meshes) - 1

        def wait(self, rid, timeout=-1.0):
            rep = {"status": 0, "outer_iters": 3, "cg_iters": 10}
            return FakeInstance(self.meshes[rid]), rep, 0.01

        def close(self):
            pass

    cp.Server = FakeServer
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out[rank] = bench.sharded_service_leg(0, rank, world, dist, n_requests=4)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("fail_rank", [-1, 1])
def test_bench_sharded_leg_on_two_gloo_ranks(fail_rank):
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_bench_shard_rank, args=(2, port, fail_rank, out), nprocs=2, join=True)
        res = dict(out)
    if fail_rank >= 0:
        # both ranks finish (no collective left waiting) and report the failure
        assert "rank 1: RuntimeError('service failed to start')" in res[0]["error"]
        assert res[0] == res[1]
        return
    r0 = res[0]
    assert r0["requests"] == 4 and r0["ranks"] == 2 and r0["statuses"] == [0]
    shares = sorted(i for s in r0["shares"] for i in s["requests"])
    assert shares == [0, 1, 2, 3]
    # checksum = sum |u| of the stand-in result, 0.5 per DOF
    from cudaplasticity_b200 import workload

    dofs = [workload.instance(i, seed=20261203)["params"]["dof"] for i in range(4)]
    assert r0["checksums"] == pytest.approx([0.5 * d for d in dofs])
