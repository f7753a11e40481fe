"""GPU tests of the batched mixed-precision engine (cp_batch_*), through the
C ABI.

Bars: every instance of a batch within 1e-8 of the reference's FP64 golden
state (the same bar as the single-instance mixed mode) with the identical
yielded set; an instance's result bit-identical whether it runs alone or in
a mix of other instances, and whether it joined at the start or while the
others were already running (every cross-tile sum is reduced per instance in
a fixed order); per-instance failures stay per instance."""
import os

import numpy as np
import pytest

import cudaplasticity_b200 as cp
import product_runner
import scenarios
from cudaplasticity_b200 import workload
from parity import field_error, yielded

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-8
BATCH_KW = dict(aitken=1, adaptive_cg=1, inner_tol=1e-3)
CHECK = ["uv", "sig_i", "eps_p_i", "exx", "sxx", "psi"]


@pytest.fixture(scope="module")
def ctx():
    c = cp.Context(0)
    yield c
    c.close()


def scenario_instance(ctx, name, workdir):
    m, lines = scenarios.scenario_lines(name, os.path.join(workdir, f"{name}.bin"))
    job, (rp, mask, uv) = product_runner.build_inputs(lines, m)
    inst = cp.Instance(ctx, m, product_runner.material_of(job))
    inst.set_loads(rp, mask, uv)
    kw = dict(cg_tol=job["cg_eps"], outer_tol=job["outer_eps"], max_outer=job["max_outer"], levels=job["levels"],
              max_cg=2_000_000, **BATCH_KW)
    return inst, kw


def workload_instance(ctx, i, **gen):
    w = workload.instance(i, **gen)
    inst = cp.Instance(ctx, w["mesh"], w["material"])
    inst.set_loads(w["rp"], w["mask"], w["uv"])
    # bit-identity does not need a tight outer tolerance; the cap keeps the
    # slowly converging (heavily plastic) seeds short
    kw = dict(cg_tol=1e-10, outer_tol=1e-6, max_outer=120, levels=w["levels"], max_cg=2_000_000, precond=1,
              **BATCH_KW)
    return inst, kw


def run_all(batch):
    out = {}
    while True:
        active, done = batch.run()
        for slot, inst, rep in batch.harvest():
            out[id(inst)] = (inst, rep)
        if active == 0:
            return out


@pytest.mark.parametrize("names", [("hole12_pow", "ogrid16_bilin", "ogrid16_hollomon", "ring_pw")])
def test_batch_matches_fp64_reference(names, ctx, golden_dir, workdir):
    """Four reference scenarios of different sizes, diagrams and load-level
    counts in one batch; each within 1e-8 of its FP64 golden state."""
    b = cp.Batch(ctx, max_instances=8)
    insts = {}
    for n in names:
        inst, kw = scenario_instance(ctx, n, workdir)
        b.add(inst, **kw)
        insts[n] = inst
    res = run_all(b)
    for n in names:
        inst, rep = res[id(insts[n])]
        assert rep["status"] == 0, (n, rep)
        assert rep["levels_done"] == scenarios.SCENARIOS[n].get("levels", 1)
        g = dict(np.load(os.path.join(golden_dir, f"{n}.npz")))
        st = inst.state()
        for k in ["uv", "sig_i", "eps_p_i"]:
            assert field_error(k, st, g) <= MIXED_TOL, (n, k, field_error(k, st, g))
        assert np.array_equal(yielded(st, 1e-9), yielded(g, 1e-9)), n
        assert rep["cg_iters"] > 0 and rep["fp64_spmv"] > 0 and rep["seconds"] > 0
        inst.close()
    b.close()


def test_batch_with_8_node_instances(ctx, golden_dir, workdir):
    """8-node (Q8) instances next to a 4-node one: the batch switches to the
    kernels with the 8-node element when the first joins; every instance
    within 1e-8 of its FP64 golden state, and the 4-node instance bit-identical
    to its run in a batch without 8-node instances."""
    names = ("hole12_q8_pow", "ring_q8_pw", "hole12_pow")
    b0 = cp.Batch(ctx, max_instances=2, max_width=24)
    inst, kw = scenario_instance(ctx, "hole12_pow", workdir)
    b0.add(inst, **kw)
    (inst0, _), = run_all(b0).values()
    q4_alone = inst0.state()
    inst0.close()
    b0.close()
    b = cp.Batch(ctx, max_instances=4, max_width=24)
    insts = {}
    for n in names:
        inst, kw = scenario_instance(ctx, n, workdir)
        b.add(inst, **kw)
        insts[n] = inst
    res = run_all(b)
    for n in names:
        inst, rep = res[id(insts[n])]
        assert rep["status"] == 0, (n, rep)
        g = dict(np.load(os.path.join(golden_dir, f"{n}.npz")))
        st = inst.state()
        for k in ["uv", "sig_i", "eps_p_i"]:
            assert field_error(k, st, g) <= MIXED_TOL, (n, k, field_error(k, st, g))
        assert np.array_equal(yielded(st, 1e-9), yielded(g, 1e-9)), n
        if n == "hole12_pow":
            for k in cp.FIELDS + ["uv"]:
                assert np.array_equal(st[k], q4_alone[k]), k
        inst.close()
    b.close()


def test_batch_agrees_with_single_instance_mixed_solve(ctx, workdir):
    """Same algorithm as cp_solve in mixed precision: the batched result of an
    instance agrees with the single-instance solve to the mixed bar."""
    inst, kw = scenario_instance(ctx, "ring_pw", workdir)
    b = cp.Batch(ctx, max_instances=2)
    b.add(inst, **kw)
    (inst_b, rep_b), = run_all(b).values()
    got = inst_b.state()
    inst_b.close()
    single, kw = scenario_instance(ctx, "ring_pw", workdir)
    rep_s = single.solve(precision=cp.CP_PREC_MIXED, **kw)
    ref = single.state()
    single.close()
    for k in CHECK:
        assert field_error(k, got, ref) <= MIXED_TOL, (k, field_error(k, got, ref))
    # the linear solves differ (residual replacement here, restarts in the
    # single-instance mode), so the outer paths may differ by a few iterations
    assert abs(rep_b["outer_iters"] - rep_s["outer_iters"]) <= max(3, rep_s["outer_iters"] // 4)
    b.close()


def test_result_identical_alone_and_in_the_mix(ctx):
    """Seeded workload instances (plates and rings, piecewise diagrams,
    uneven sizes): each solved alone and inside a mix, bit-identical."""
    gen = dict(dof_min=600, dof_max=6000)
    ids = list(range(6))
    alone = {}
    for i in ids:
        inst, kw = workload_instance(ctx, i, **gen)
        b = cp.Batch(ctx, max_instances=1)
        b.add(inst, **kw)
        (inst_b, rep), = run_all(b).values()
        alone[i] = (inst_b.state(), rep)
        inst_b.close()
        b.close()
    b = cp.Batch(ctx, max_instances=8)
    mine = {}
    for i in ids:
        inst, kw = workload_instance(ctx, i, **gen)
        b.add(inst, **kw)
        mine[id(inst)] = i
    res = run_all(b)
    assert len(res) == len(ids)
    for key, (inst, rep) in res.items():
        i = mine[key]
        st = inst.state()
        ref, rep_a = alone[i]
        assert rep["status"] == rep_a["status"]
        for k in cp.FIELDS + ["uv"]:
            assert np.array_equal(st[k], ref[k]), (i, k)
        assert rep["outer_iters"] == rep_a["outer_iters"] and rep["cg_iters"] == rep_a["cg_iters"]
        inst.close()
    b.close()


def test_instances_join_a_running_batch(ctx):
    """Continuous batching: the batch runs until one instance finishes, the
    finished one is harvested and a new one joins while the rest are mid-solve;
    every result equals its solve alone."""
    gen = dict(dof_min=600, dof_max=6000)
    order = [10, 11, 12, 13, 14]
    alone = {}
    for i in order:
        inst, kw = workload_instance(ctx, i, **gen)
        b = cp.Batch(ctx, max_instances=1)
        b.add(inst, **kw)
        (inst_b, rep), = run_all(b).values()
        alone[i] = inst_b.state()
        inst_b.close()
        b.close()
    b = cp.Batch(ctx, max_instances=3)
    pending = list(order)
    which = {}
    finished = {}
    for _ in range(2):
        inst, kw = workload_instance(ctx, pending[0], **gen)
        b.add(inst, **kw)
        which[id(inst)] = pending.pop(0)
    joined_mid_run = 0
    while which:
        active, done = b.run(any_done=True, max_trips=50)
        for slot, inst, rep in b.harvest():
            assert rep["status"] in (0, cp._capi.CP_ERR_NOT_CONVERGED)
            finished[which.pop(id(inst))] = inst.state()
            inst.close()
        while pending and len(which) < 3:
            inst, kw = workload_instance(ctx, pending[0], **gen)
            b.add(inst, **kw)
            which[id(inst)] = pending.pop(0)
            joined_mid_run += active > 0
    assert joined_mid_run >= 1
    for i in order:
        for k in ["uv", "sig_i", "psi", "eps_p_i"]:
            assert np.array_equal(finished[i][k], alone[i][k]), (i, k)
    b.close()


def test_per_instance_failure_stays_per_instance(ctx, workdir):
    """An instance that hits its outer-iteration cap reports
    CP_ERR_NOT_CONVERGED; the others in the batch are unaffected."""
    b = cp.Batch(ctx, max_instances=4)
    ok, kw = scenario_instance(ctx, "hole12_pow", workdir)
    capped, kw2 = scenario_instance(ctx, "hole12_lin", workdir)
    kw2["max_outer"] = 2
    b.add(ok, **kw)
    b.add(capped, **kw2)
    with pytest.raises(cp.CuplastError) as e:
        capped.solve()
    assert e.value.status == cp._capi.CP_ERR_BUSY  # owned by the batch
    res = run_all(b)
    assert res[id(ok)][1]["status"] == 0
    assert res[id(capped)][1]["status"] == cp._capi.CP_ERR_NOT_CONVERGED
    assert res[id(capped)][1]["outer_iters"] == 2
    ok.close()
    capped.close()
    b.close()


def test_batch_rejects_fp64_and_unset_loads(ctx, workdir):
    b = cp.Batch(ctx, max_instances=2)
    inst, kw = scenario_instance(ctx, "hole12_pow", workdir)
    o = cp.solve_opts(**dict(kw, precision=cp.CP_PREC_FP64))
    import ctypes

    slot = ctypes.c_int()
    st = cp._capi.lib().cp_batch_add(b._h, inst._h, ctypes.byref(o), ctypes.byref(slot))
    assert st == cp._capi.CP_ERR_UNSUPPORTED
    bare = cp.Instance(ctx, scenarios.SCENARIOS["hole12_pow"]["mesh"](), cp.material(1000.0))
    with pytest.raises(cp.CuplastError):
        b.add(bare, **kw)
    bare.close()
    inst.close()
    b.close()


def test_autotuner_keeps_results(ctx):
    """The autotuner times tile sizes per size bucket without changing any
    instance's state: results equal the untuned batch's."""
    gen = dict(dof_min=600, dof_max=20000)
    ids = [20, 21, 22, 23]
    results = []
    for tune in (False, True):
        b = cp.Batch(ctx, max_instances=8)
        mine = {}
        for i in ids:
            inst, kw = workload_instance(ctx, i, **gen)
            b.add(inst, **kw)
            mine[id(inst)] = i
        if tune:
            b.run(max_trips=3)  # mid-solve: instances in various phases
            ms = b.autotune()
            assert ms > 0
        res = run_all(b)
        results.append({mine[k]: inst.state() for k, (inst, rep) in res.items()})
        for inst, _ in res.values():
            inst.close()
        b.close()
    for i in ids:
        assert np.array_equal(results[0][i]["uv"], results[1][i]["uv"]), i


def test_instance_can_join_again_after_harvest(ctx):
    """A harvested instance can be reset and added again (its batch buffers
    are reused); the second solve repeats the first bit for bit."""
    inst, kw = workload_instance(ctx, 3, dof_min=600, dof_max=6000)
    w = workload.instance(3, dof_min=600, dof_max=6000)
    b = cp.Batch(ctx, max_instances=2)
    runs = []
    for _ in range(2):
        inst.reset_state()
        inst.set_loads(w["rp"], w["mask"], w["uv"])
        b.add(inst, **kw)
        (got, rep), = run_all(b).values()
        assert got is inst
        runs.append((inst.state(), rep))
    for k in cp.FIELDS + ["uv"]:
        assert np.array_equal(runs[0][0][k], runs[1][0][k]), k
    assert runs[0][1]["cg_iters"] == runs[1][1]["cg_iters"]
    inst.close()
    b.close()
