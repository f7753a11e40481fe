"""GPU tests of the solve service (cp_server_*), through the C ABI.

Requests arrive from a separate thread at random times while others are on
the device (continuous batching); each result must be bit-identical to the
same request solved alone, admission must respect the byte budget, and a
request larger than the budget is rejected at submission. FP64 requests run
on the service's lanes (cp_solve, several at once) and equal cp_solve alone."""
import random
import threading
import time

import numpy as np
import pytest

import cudaplasticity_b200 as cp
from cudaplasticity_b200 import workload

pytestmark = pytest.mark.gpu

GEN = dict(dof_min=600, dof_max=6000)
# Some seeded requests converge slowly (heavy plasticity); the cap keeps the
# test short, and a capped request must still equal its capped solve alone.
KW = dict(cg_tol=1e-10, outer_tol=1e-7, max_outer=120, max_cg=2_000_000, precond=1, aitken=1, adaptive_cg=1,
          inner_tol=1e-3)


def alone(ctx, w):
    inst = cp.Instance(ctx, w["mesh"], w["material"])
    inst.set_loads(w["rp"], w["mask"], w["uv"])
    b = cp.Batch(ctx, max_instances=1)
    b.add(inst, levels=w["levels"], **KW)
    while b.run()[0]:
        pass
    (_, inst_b, rep), = b.harvest()
    st = inst_b.state()
    inst_b.close()
    b.close()
    return st, rep


def submit_all(server, ws, rate_hz, seed=7):
    """Submits the requests from a thread at Poisson arrival times; returns ids."""
    ids = [None] * len(ws)
    rng = random.Random(seed)

    def run():
        for k, w in enumerate(ws):
            time.sleep(rng.expovariate(rate_hz))
            ids[k] = server.submit(w["mesh"], w["material"], w["rp"], w["mask"], w["uv"], levels=w["levels"], **KW)

    t = threading.Thread(target=run)
    t.start()
    return t, ids


def test_served_results_equal_alone():
    ws = [workload.instance(i, increments=(1, 3), **GEN) for i in range(30, 38)]
    ctx = cp.Context(0)
    ref = [alone(ctx, w) for w in ws]
    srv = cp.Server(max_inflight=4)
    try:
        t, ids = submit_all(srv, ws, rate_hz=200.0)
        t.join()
        lat = []
        for k, rid in enumerate(ids):
            inst, rep, latency = srv.wait(rid, timeout=300.0)
            assert rep["status"] == ref[k][1]["status"], (rep, ref[k][1])
            st = inst.state()
            for f in cp.FIELDS + ["uv"]:
                assert np.array_equal(st[f], ref[k][0][f]), (k, f)
            assert rep["outer_iters"] == ref[k][1]["outer_iters"] and rep["cg_iters"] == ref[k][1]["cg_iters"]
            lat.append(latency)
            inst.close()
        s = srv.stats()
        assert s["completed"] == len(ws) and s["admitted"] == len(ws)
        assert s["runs"] >= 2 and all(x > 0 for x in lat)
    finally:
        srv.close()
        ctx.close()


def test_admission_respects_byte_budget():
    ws = [workload.instance(i, **GEN) for i in range(40, 46)]
    fps = [cp.footprint(w["mesh"], cp.CP_PREC_MIXED) for w in ws]
    budget = int(1.5 * max(fps))
    ctx = cp.Context(0)
    ref = [alone(ctx, w) for w in ws]
    srv = cp.Server(max_bytes=budget)
    try:
        ids = [srv.submit(w["mesh"], w["material"], w["rp"], w["mask"], w["uv"], levels=w["levels"], **KW)
               for w in ws]
        for k, rid in enumerate(ids):
            inst, rep, _ = srv.wait(rid, timeout=300.0)
            assert rep["status"] == ref[k][1]["status"]
            assert np.array_equal(inst.field("uv"), ref[k][0]["uv"])
            inst.close()
        s = srv.stats()
        assert 0 < s["peak_bytes"] <= budget
        assert s["completed"] == len(ws)
        with pytest.raises(cp.CuplastError) as e:
            big = workload.instance(0)  # far above the budget
            srv.submit(big["mesh"], big["material"], big["rp"], big["mask"], big["uv"], **KW)
        assert e.value.status == cp._capi.CP_ERR_NOMEM
        assert srv.stats()["rejected"] == 1
    finally:
        srv.close()
        ctx.close()


def test_destroy_with_requests_in_flight_returns():
    ws = [workload.instance(i, **GEN) for i in range(50, 54)]
    srv = cp.Server(max_inflight=2)
    for w in ws:
        srv.submit(w["mesh"], w["material"], w["rp"], w["mask"], w["uv"], levels=w["levels"], **KW)
    t0 = time.time()
    srv.close()
    assert time.time() - t0 < 60.0


FP64_KW = dict(cg_tol=1e-10, outer_tol=1e-7, max_outer=120, max_cg=2_000_000, precond=1, aitken=1, adaptive_cg=1)


def alone_fp64(ctx, w):
    inst = cp.Instance(ctx, w["mesh"], w["material"])
    inst.set_loads(w["rp"], w["mask"], w["uv"])
    rep = inst.solve(allow_not_converged=True, levels=w["levels"], **FP64_KW)
    st = inst.state()
    inst.close()
    return st, rep


def test_fp64_lanes_equal_cp_solve_alone_next_to_the_batch():
    """FP64 requests are solved by cp_solve on the server's lanes, several at
    once on their own streams, while mixed requests join the batch: every
    FP64 result is bit-identical to the same request solved alone with
    cp_solve, and every mixed one has the status it has alone."""
    ws = [workload.instance(i, increments=(1, 3), **GEN) for i in range(60, 68)]
    ctx = cp.Context(0)
    kinds = ["fp64" if k % 4 != 3 else "mixed" for k in range(len(ws))]
    ref = [alone_fp64(ctx, w) if kind == "fp64" else alone(ctx, w) for w, kind in zip(ws, kinds)]
    srv = cp.Server(fp64_lanes=4)
    try:
        ids = []
        for w, kind in zip(ws, kinds):
            kw = dict(FP64_KW, precision=cp.CP_PREC_FP64) if kind == "fp64" else KW
            ids.append(srv.submit(w["mesh"], w["material"], w["rp"], w["mask"], w["uv"], levels=w["levels"], **kw))
        for k, rid in enumerate(ids):
            inst, rep, latency = srv.wait(rid, timeout=600.0)
            assert rep["status"] == ref[k][1]["status"], (k, rep, ref[k][1])
            if kinds[k] == "fp64":
                st = inst.state()
                for f in cp.FIELDS + ["uv"]:
                    assert np.array_equal(st[f], ref[k][0][f]), (k, f)
                assert rep["cg_iters"] == ref[k][1]["cg_iters"] and rep["outer_iters"] == ref[k][1]["outer_iters"]
            assert latency > 0
            inst.close()
        assert srv.stats()["completed"] == len(ws)
    finally:
        srv.close()
        ctx.close()


def test_results_read_while_lanes_start_their_next_requests():
    """Requests larger than one thread-block cluster holds run the graph-loop
    CG, whose first solve on an instance captures a CUDA graph on the lane's
    stream. The caller reads each result (every field, device to host) as
    soon as it completes, while the two lanes already set up and capture the
    next requests: every read succeeds and equals cp_solve alone bit for bit
    (the outer cap keeps the test short; capped results compare too)."""
    gen = dict(dof_min=20000, dof_max=40000)
    kw = dict(FP64_KW, max_outer=3)
    ws = [workload.instance(i, **gen) for i in range(80, 88)]
    ctx = cp.Context(0)
    ref = []
    for w in ws:
        inst = cp.Instance(ctx, w["mesh"], w["material"])
        inst.set_loads(w["rp"], w["mask"], w["uv"])
        rep = inst.solve(allow_not_converged=True, levels=w["levels"], **kw)
        ref.append((inst.state(), rep))
        inst.close()
    srv = cp.Server(fp64_lanes=2)
    try:
        ids = [srv.submit(w["mesh"], w["material"], w["rp"], w["mask"], w["uv"], levels=w["levels"],
                          precision=cp.CP_PREC_FP64, **kw) for w in ws]
        for k, rid in enumerate(ids):
            inst, rep, _ = srv.wait(rid, timeout=600.0)
            st = inst.state()
            inst.close()
            assert rep["status"] == ref[k][1]["status"], (k, rep)
            for f in cp.FIELDS + ["uv"]:
                assert np.array_equal(st[f], ref[k][0][f]), (k, f)
    finally:
        srv.close()
        ctx.close()


def test_destroy_with_fp64_solves_in_flight_returns():
    """Closing the server cancels the lanes' solves at their next outer
    iteration and the requests still queued."""
    ws = [workload.instance(i, **GEN) for i in range(70, 76)]
    srv = cp.Server(fp64_lanes=2)
    for w in ws:
        srv.submit(w["mesh"], w["material"], w["rp"], w["mask"], w["uv"], levels=w["levels"],
                   precision=cp.CP_PREC_FP64, **FP64_KW)
    time.sleep(0.5)
    t0 = time.time()
    srv.close()
    assert time.time() - t0 < 60.0


def test_sharded_shares_equal_requests_solved_alone():
    """The instance sharding of cudaplasticity_b200.shard, its two shares run
    one after the other through one service (what two ranks do on two GPUs):
    every request is solved once, and its result equals the same request
    solved alone with cp_solve, bit for bit."""
    from cudaplasticity_b200 import shard

    ws = [workload.instance(i, increments=(1, 3), **GEN) for i in range(80, 86)]
    ctx = cp.Context(0)
    ref = [alone_fp64(ctx, w) for w in ws]
    parts = shard.partition([shard.request_cost(w["params"]["dof"], w["levels"]) for w in ws], 2)
    assert sorted(parts[0] + parts[1]) == list(range(len(ws))) and parts[0] and parts[1]
    srv = cp.Server(fp64_lanes=3)
    results = {}
    try:
        def submit(w):
            return srv.submit(w["mesh"], w["material"], w["rp"], w["mask"], w["uv"], levels=w["levels"],
                              precision=cp.CP_PREC_FP64, **FP64_KW)

        def wait(rid):
            inst, rep, latency = srv.wait(rid, timeout=600.0)
            results[rid] = (inst.state(), rep)
            inst.close()
            return {"status": rep["status"], "latency": latency, "rid": rid}

        recs = [shard.run_share(p, lambda i: ws[i], submit, wait) for p in parts]
    finally:
        srv.close()
        ctx.close()
    merged = shard.merge_records(recs)
    summ = shard.summarize(merged, len(ws), 2)
    assert summ["requests"] == len(ws) and summ["seconds"] > 0
    for k in range(len(ws)):
        st, rep = results[merged[k]["rid"]]
        assert rep["status"] == ref[k][1]["status"], (k, rep, ref[k][1])
        for f in cp.FIELDS + ["uv"]:
            assert np.array_equal(st[f], ref[k][0][f]), (k, f)
        assert rep["cg_iters"] == ref[k][1]["cg_iters"]
