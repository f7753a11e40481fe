"""Benchmark: converged plastic solves per second on one B200 (per GPU, replicas).

Workload (the plain method on the small plate, which the reference's CPU path
runs): plane-stress 200 x 200 mm plate with a centred 20 mm hole, O-grid of 64
circumferential x 64 radial quads (4160 nodes, 8320 DOF), E = 210 GPa, nu = 0.3,
bilinear hardening sigma_y = 250 MPa, E_t = 2 GPa; 200 MPa traction on the top
edge in 10 equal increments; bottom edge fixed in y, bottom-left node fixed;
CG tolerance 1e-10, outer (secant) tolerance 1e-6. Quads on the O-grid nodes:
the reference has no triangle element. Synthetic, seeded-free (deterministic).

One step = one complete solve (all 10 load levels to convergence). The product
arm runs the FP64 drop-in path (one launch per CG iteration; Aitken-relaxed
secant iteration, block-Jacobi
PCG with the linear tolerance following the outer error; same fixed point as
the reference). ``--impl reference`` runs the reference implementation's own
CPU path (oracle/_ref/cpref, built from its sources) on the same job with all
host cores.

Beside the headline, the line carries:
  error_vs_reference  the timed result against the reference CPU path's
           result on the same job;
  roofline (CG GB/s)  the FP64 CG iteration of the 2.1M-DOF plate (k_f_iter),
           CUDA events, against the measured HBM copy peak; the FP32 SpMV
           beside it;
  served_vs_plain  the metric's comparison: the first requests of the
           seeded batch stream (cudaplasticity_b200/workload.py: DOF
           log-uniform in [2k, 200k], plates and rings, 5-segment diagrams)
           solved one at a time through the plain FP64 drop-in, and through
           the solve service (cp_server, FP64 lanes) under Poisson arrivals
           at 10, 100 and 1000 requests/s: solves/s, p50/p99 latency and each
           result's error against the plain FP64 result;
  batched  closed-loop saturation throughput of the batched mixed-precision
           engine (512 resident batch-stream instances) and its CG
           iteration's live roofline;
  config2  configuration 2 end to end: the 2.1M-DOF Hollomon plate, 20
           increments, through the drop-in, and the reference-composed CPU
           per-iteration rate on the same mesh.

Multi-GPU: the path does not shard (one solve is one small instance), so N GPUs
run N independent replicas ("replicas only"); value = solves of all ranks /
max-over-ranks time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(workload="hole_plate_ogrid64x64_q4_8320dof", plate_mm=200, hole_radius_mm=20, n_circ=64, n_rad=64,
                nodes=4160, dof=8320, elements=4096, E_mpa=210000, nu=0.3, sigma_y=250, E_t=2000, traction_mpa=200,
                increments=10, cg_tol=1e-10, outer_tol=1e-6)
SOLVE_KW = dict(cg_tol=1e-10, outer_tol=1e-6, max_outer=2000, levels=10, aitken=1, adaptive_cg=2, precond=1,
                max_cg=2_000_000, predict=1, recycle=6)
PRECOND_NAMES = {0: "unpreconditioned CG", 1: "block-Jacobi PCG", 2: "aggregation-multigrid V-cycle PCG"}
METRIC = "converged solves/s (200 mm plate, 20 mm hole, 64x64 O-grid, 8320 DOF, FP64, <=1e-6 outer / 1e-10 CG)"


def build_problem():
    import cudaplasticity_b200 as cp

    mesh = cp.Mesh.rect_with_hole(-100.0, 100.0, -100.0, 100.0, 20.0, 16, 16, rad_n=64)
    loads = cp.Loads().set_force(2, 0.0, 200.0).fix_border_hor(0).fix_point(-100.0, -100.0)
    rp, mask, uv = loads.build(mesh)
    mat = cp.material(210000.0, 0.3, diagram="linear", sigma_t=250.0, k_t=2000.0)
    return mesh, mesh.arrays(), mat, rp, mask, uv


def reference_mesh():
    """The same O-grid for the CPU arms, from the numpy restatement of the
    reference's generator (tests/meshgen.py; digest-pinned to
    Mesh::genRectWithHole), so that the reference arm maps no product code."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import meshgen

    return meshgen.hole_plate(-100.0, 100.0, -100.0, 100.0, 20.0, 16, 16, rad_n=64)


def reference_job_lines(mesh_path):
    return ["mode phases", f"mesh file {mesh_path}", "levels 10", "cg_eps 1e-10", "outer_eps 1e-6",
            "max_outer 100000", "diagram linear 210000 250 2000", "material 210000 0.3 1", "force 2 0 200 0",
            "fixborderhor 0", "fixpoint -100 -100"]


def line_config(world):
    """The `config` of both arms' lines (identical for the same N)."""
    return dict(WORKLOAD, parallelism=f"replicas x{world}",
                l2="GPU arm: 512 MB written between steps (L2 flushed); CPU arm: no flush")


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, gpu):
        self.gpu = gpu
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                vals = [v.strip() for v in out.stdout.strip().split(",")]
                if len(vals) == 7:
                    self.samples.append(vals)
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[3 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_baseline_run(threads=None, first_level_only=False):
    """The reference's own CPU path on the same job (oracle/_ref/cpref), or the
    oracle restatement where the reference could not be built. With
    first_level_only, the job's first load increment alone (20 MPa, one
    level): the warm-up of the reference arm."""
    import tempfile

    import oracle

    threads = threads or os.cpu_count()
    arrays = reference_mesh()
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "m.bin")
        oracle.write_mesh(path, arrays["node_xy"], elem4=arrays["elem4"], borders=arrays["borders"])
        lines = reference_job_lines(path)
        if first_level_only:
            lines = [("levels 1" if ln.startswith("levels") else "force 2 0 20 0" if ln.startswith("force") else ln)
                     for ln in lines]
        t0 = time.perf_counter()
        if oracle.have_reference():
            r = oracle.run_reference(lines, threads=threads)
            kind = "reference"
        else:
            os.environ["OMP_NUM_THREADS"] = str(threads)
            r = oracle.run_oracle(lines)
            kind = "port"
        wall = time.perf_counter() - t0
    return dict(seconds=wall, kind=kind, cores=threads, outer=int(r["outer_per_level"].sum()),
                cg=int(r["cg_per_level"].sum()), state=r)


def run_reference_arm(args):
    rank, world, local = dist_env()
    if rank != 0:
        return
    steps = []
    for _ in range(max(0, args.warmup)):
        # the first load increment of the same job: pages in the harness and
        # the job's mesh, starts the OpenMP thread pool
        cpu_baseline_run(first_level_only=True)
    info = None
    for _ in range(args.steps):
        info = cpu_baseline_run()
        steps.append(info["seconds"])
    total = sum(steps)
    value = len(steps) / total
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(steps),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": line_config(1),
            "solver": "reference CPU path (oracle/_ref/cpref, built from the reference sources): its own phases "
                      "(fillGlobalStiffness, ConjGradSolver::solve, updateParameters, exitCondition) driven per load "
                      "level by the harness with the job's tolerances instead of solve()'s fixed 1e-7 / 1e-5; "
                      "unpreconditioned CG, plain secant iteration",
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": info["cores"], "kind": info["kind"],
                             "sample": "full 8320-DOF hole-plate solve (10 levels, CG 1e-10, outer 1e-6) per step, "
                                       "reference CPU path through its phase functions, all host cores; warm-up "
                                       "steps solve the first increment only"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "detail": {"outer_iters": info["outer"], "cg_iters": info["cg"]}}
    print(json.dumps(line), flush=True)


def error_vs_reference(state, ref, tight):
    """The timed solve's result against the reference CPU path's result on the
    same job (both stopped at outer 1e-6 / CG 1e-10, by different iterations),
    and the reference's own distance from the tight FP64 fixed point, which
    bounds what agreement the shared tolerances allow."""
    import numpy as np

    def rel(a, b):
        nb = np.linalg.norm(b)
        return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / nb) if nb > 0 else 0.0

    ours_y = np.asarray(state["psi"]) > 1.0 + 1e-12
    ref_y = np.asarray(ref["psi"]) > 1.0 + 1e-12
    tight_y = np.asarray(tight["psi"]) > 1.0 + 1e-12
    return {"rel_l2": {k: rel(state[k], ref[k]) for k in ("uv", "sig_i", "eps_p_i")},
            "reference_vs_tight_fp64": {k: rel(ref[k], tight[k]) for k in ("uv", "sig_i", "eps_p_i")},
            "yielded": int(ours_y.sum()), "yielded_reference": int(ref_y.sum()),
            "yielded_sets_identical": bool(np.array_equal(ours_y, ref_y)),
            "yielded_differ": int((ours_y != ref_y).sum()),
            "yielded_sets_identical_at_tight_fp64": bool(np.array_equal(tight_y, ref_y))}


def flush_l2(ctx_dev):
    """Writes 512 MB (4x the 126 MB L2) so the next step starts cold."""
    import torch

    buf = getattr(flush_l2, "buf", None)
    if buf is None:
        buf = flush_l2.buf = torch.empty(64 * 1024 * 1024, dtype=torch.float64, device=f"cuda:{ctx_dev}")
    buf.fill_(1.0)
    torch.cuda.synchronize(ctx_dev)



BATCH_KW = dict(cg_tol=1e-10, outer_tol=1e-6, max_outer=2000, max_cg=5_000_000, precond=1, aitken=1, adaptive_cg=1,
                inner_tol=1e-3)
# the FP64 lanes of the solve service: the same tolerances in FP64
FP64_SERVE_KW = dict(cg_tol=1e-10, outer_tol=1e-6, max_outer=2000, max_cg=5_000_000, precond=1, aitken=1,
                     adaptive_cg=1, recycle=6)


def batched_leg(ctx, window_s=20.0, warm_s=3.0, slots=512, pool_size=768, seed=20261203):
    """The batched engine on the batch stream (512 seeded instances, DOF 2k-200k).

    saturation: closed loop, a batch of `slots` resident instances refilled
        from the stream as solves finish; converged solves per second over a
        window, and the SpMV sweep over all resident instances (CG GB/s).
        Quick requests finish first, so this is a throughput, not a comparison.
    The like-for-like comparison with the plain drop-in is compare_leg.
    """
    import numpy as np

    import cudaplasticity_b200 as cp
    from cudaplasticity_b200 import workload

    def make(i):
        w = workload.instance(i, seed=seed)
        inst = cp.Instance(ctx, w["mesh"], w["material"])
        inst.set_loads(w["rp"], w["mask"], w["uv"])
        return w, inst

    # --- saturation ---
    pool = [make(i) for i in range(pool_size)]
    b = cp.Batch(ctx, max_instances=slots)
    nxt = 0
    for _ in range(slots):
        b.add(pool[nxt][1], levels=1, **BATCH_KW)
        nxt += 1
    b.run(max_trips=2)
    ms_sweep = b.autotune()
    blocks = nodes = 0
    for _, inst in pool[:slots]:
        n, ne, nnz, nadj = inst.sizes()
        blocks += nnz // 4
        nodes += n
    # algorithmic bytes of one SpMV sweep (P phase, FP32): 4 values + one
    # column per 2x2 block, read r (or s) and z, write z' and K z'
    bytes_sweep = blocks * 20 + nodes * 4 * 8
    by_inst = {id(p[1]): p for p in pool}
    done = []
    t0 = time.perf_counter()
    t_start = None
    while True:
        now = time.perf_counter() - t0
        if t_start is None and now >= warm_s:
            t_start, launches_start = now, b.stats()["kernel_launches"]
        if now >= warm_s + window_s:
            break
        b.run(max_trips=200)
        for slot, inst, rep in b.harvest():
            done.append((time.perf_counter() - t0, by_inst[id(inst)], rep))
            if nxt < len(pool):
                b.add(pool[nxt][1], levels=1, **BATCH_KW)
                nxt += 1
    t_end = time.perf_counter() - t0
    counted = [d for d in done if d[0] > t_start]
    launches_sat = b.stats()["kernel_launches"] - launches_start
    b.close()  # releases the instances still in flight (not counted)
    for _, inst in pool:
        inst.close()
    saturation = {
        "slots": slots, "window_s": round(t_end - t_start, 2), "completed": len(counted),
        "solves_per_s": len(counted) / (t_end - t_start), "statuses": sorted({d[2]["status"] for d in counted}),
        "mean_dof_completed": float(sum(d[1][0]["params"]["dof"] for d in counted) / max(1, len(counted))),
        "resident_dof": int(2 * nodes), "gpu_launches": int(launches_sat),
        "spmv_sweep": {"ms": ms_sweep, "bytes": bytes_sweep, "gbs": bytes_sweep / (ms_sweep * 1e-3) / 1e9,
                       "kernel": "k_batch_cg P phase (autotuner probe), all resident instances"},
    }

    return {
        "workload": "batch stream: seeded instances (base seed %d), DOF log-uniform [2k, 200k], plates / rings, "
                    "5-segment piecewise diagrams, 1 load level, CG 1e-10, outer 1e-6; batched = mixed precision, "
                    "plain = FP64 drop-in one request at a time, same solver options" % seed,
        "saturation": saturation,
    }


def compare_leg(ctx, n_requests, max_outer=100, seed=20261203, lanes=8, mg=False):
    """Like for like: the plain FP64 drop-in solves the first n requests of
    the batch stream (DOF 2k-200k) one at a time; the batched mixed-precision engine
    then solves exactly the same requests (fresh instances) to completion, and
    so does the solve service's FP64 lanes, once with the block-Jacobi PCG of
    the plain run and (mg) once with the multigrid-preconditioned CG.
    Same solver options and caps for both, wall clock for both, and the error
    of each mixed-precision result against its FP64 result. Requests that hit
    the outer cap count as solved by both (same cap) and are listed."""
    import numpy as np

    import cudaplasticity_b200 as cp
    from cudaplasticity_b200 import workload

    kw = dict(BATCH_KW, max_outer=max_outer)

    def make(i):
        w = workload.instance(i, seed=seed)
        inst = cp.Instance(ctx, w["mesh"], w["material"])
        inst.set_loads(w["rp"], w["mask"], w["uv"])
        return w, inst

    plain, t_plain = {}, 0.0
    for k in range(n_requests):
        w, inst = make(k)
        t1 = time.perf_counter()
        rep = inst.solve(allow_not_converged=True, precision=cp.CP_PREC_FP64, levels=1, **kw)
        dt = time.perf_counter() - t1
        t_plain += dt
        plain[k] = (inst.state(), rep, w["params"]["dof"])
        inst.close()
        print(json.dumps({"compare_plain": k, "dof": w["params"]["dof"], "seconds": dt, "status": rep["status"],
                          "outer": rep["outer_iters"], "cg": rep["cg_iters"]}), flush=True)
    ids = sorted(plain)
    insts = {i: make(i)[1] for i in ids}
    b = cp.Batch(ctx, max_instances=len(ids))
    for i in ids:
        b.add(insts[i], levels=1, **kw)
    b.run(max_trips=1)
    b.autotune()  # tile sizes per size bucket of this set (state unchanged)
    reps = {}
    for slot, inst, rep in b.harvest():
        reps[id(inst)] = rep
    launches0 = b.stats()["kernel_launches"]
    t1 = time.perf_counter()
    while True:
        active, _ = b.run()
        for slot, inst, rep in b.harvest():
            reps[id(inst)] = rep
        if active == 0:
            break
    t_batch = time.perf_counter() - t1
    launches_fixed = b.stats()["kernel_launches"] - launches0
    errs = {"uv": 0.0, "sig_i": 0.0, "eps_p_i": 0.0}
    statuses = set()
    for i in ids:
        mixed = insts[i].state()
        ref = plain[i][0]
        statuses.add(reps[id(insts[i])]["status"])
        for f in errs:
            nrm = np.linalg.norm(ref[f])
            errs[f] = max(errs[f], float(np.linalg.norm(mixed[f] - ref[f]) / nrm) if nrm > 0 else 0.0)
        insts[i].close()
    b.close()
    fixed = {
        "workload": "first %d requests of the batch stream (DOF 2k-200k, base seed %d), outer cap %d, CG 1e-10, outer 1e-6"
                    % (n_requests, seed, max_outer),
        "requests": len(ids), "dof": [plain[i][2] for i in ids],
        "capped": [i for i in ids if plain[i][1]["status"] != 0],
        "plain_fp64_dropin": {"seconds": t_plain, "solves_per_s": len(ids) / t_plain,
                              "statuses": sorted({plain[i][1]["status"] for i in ids})},
        "batched_mixed": {"seconds": t_batch, "solves_per_s": len(ids) / t_batch, "statuses": sorted(statuses),
                          "gpu_launches": int(launches_fixed)},
        "speedup_vs_plain": t_plain / t_batch,
        "max_rel_err_mixed_vs_fp64": errs,
    }
    # the same requests through the solve service's FP64 lanes (cp_solve,
    # several at once): FP64 results, which must equal the plain ones
    srv = cp.Server(fp64_lanes=lanes)
    ws = {i: workload.instance(i, seed=seed) for i in ids}
    t1 = time.perf_counter()
    rids = {i: srv.submit(ws[i]["mesh"], ws[i]["material"], ws[i]["rp"], ws[i]["mask"], ws[i]["uv"], levels=1,
                          precision=cp.CP_PREC_FP64, **{k: v for k, v in kw.items() if k != "inner_tol"})
            for i in ids}
    same, lane_status = True, set()
    for i in ids:
        inst, rep, _ = srv.wait(rids[i], timeout=-1.0)
        lane_status.add(rep["status"])
        st = inst.state()
        same = same and all(np.array_equal(st[f], plain[i][0][f]) for f in ("uv", "sig_i", "eps_p_i"))
        inst.close()
    t_lanes = time.perf_counter() - t1
    srv.close()
    fixed["fp64_lanes"] = {"lanes": lanes, "seconds": t_lanes, "solves_per_s": len(ids) / t_lanes,
                           "statuses": sorted(lane_status), "identical_to_plain": bool(same),
                           "speedup_vs_plain": t_plain / t_lanes}
    if mg:
        # and once more with the multigrid-preconditioned CG on the lanes: the
        # same fixed point, reached through other iterates (error stated)
        srv = cp.Server(fp64_lanes=lanes)
        mkw = {k: v for k, v in kw.items() if k != "inner_tol"}
        mkw["precond"] = 2
        t1 = time.perf_counter()
        rids = {i: srv.submit(ws[i]["mesh"], ws[i]["material"], ws[i]["rp"], ws[i]["mask"], ws[i]["uv"],
                              levels=1, precision=cp.CP_PREC_FP64, **mkw) for i in ids}
        mg_status, mg_errs, mg_cg = set(), {"uv": 0.0, "sig_i": 0.0, "eps_p_i": 0.0}, 0
        for i in ids:
            inst, rep, _ = srv.wait(rids[i], timeout=-1.0)
            mg_status.add(rep["status"])
            mg_cg += rep["cg_iters"]
            st = inst.state()
            for f in mg_errs:
                nrm = np.linalg.norm(plain[i][0][f])
                mg_errs[f] = max(mg_errs[f], float(np.linalg.norm(st[f] - plain[i][0][f]) / nrm) if nrm > 0 else 0.0)
            inst.close()
        t_mg = time.perf_counter() - t1
        srv.close()
        fixed["fp64_lanes_multigrid"] = {"lanes": lanes, "seconds": t_mg, "solves_per_s": len(ids) / t_mg,
                                         "statuses": sorted(mg_status), "cg_iters": mg_cg,
                                         "plain_cg_iters": sum(plain[i][1]["cg_iters"] for i in ids),
                                         "max_rel_err_vs_plain": mg_errs, "speedup_vs_plain": t_plain / t_mg}
    return fixed


CONFIG2 = dict(workload="hole_plate_ogrid1024x1024_q4_2099200dof_hollomon", n_circ=1024, n_rad=1024,
               nodes=1049600, dof=2099200, elements=1048576, E_mpa=210000, nu=0.3, sigma_y=250, eps0=0.002,
               n_exp=0.2, traction_mpa=220, increments=20, cg_tol=1e-10, outer_tol=1e-6)


def config2_leg(ctx, cpu=True, cpu_cg_eps=1e-2):
    """Configuration 2 end to end: the 1024 x 1024 O-grid plate (2.1M DOF),
    Hollomon hardening sy (1 + eps_p / eps0)^n, 220 MPa in 20 increments, CG
    1e-10, outer 1e-6, one FP64 solve through the drop-in (host arrays in,
    every field out) with the headline's solver options.

    CPU baseline: the reference cannot run this mesh as shipped (its band
    matrix would take about 138 GB), so the reference-composed CSR-direct
    harness (oracle/_ref/cpref_csr, mode phases_csr: the reference's calcBs,
    initConditions, SparseSLAE, formC / formKe4, ConjGradSolver::solve,
    updateParameters, exitCondition, with the element matrices added straight
    into CSR) runs the first outer step of the first increment with a loose
    CG tolerance, on all host cores: its set-up, assembly, CG-iteration and
    update times. The CPU estimate of the full solve applies those per-step
    and per-iteration times to the GPU solve's outer and CG iteration counts
    (an estimate at equal iteration counts, not a measured CPU solve)."""
    import numpy as np

    import cudaplasticity_b200 as cp

    mesh = cp.Mesh.rect_with_hole(-100.0, 100.0, -100.0, 100.0, 20.0, 256, 256, rad_n=1024)
    arrays = mesh.arrays()
    rp, mask, uv = cp.Loads().set_force(2, 0.0, 220.0).fix_border_hor(0).fix_point(-100.0, -100.0).build(mesh)
    mat = cp.material(210000.0, 0.3, diagram="hollomon", sigma_y=250.0, eps0=0.002, n=0.2)
    kw = dict(SOLVE_KW, levels=20, max_cg=5_000_000, max_outer=20000)
    t0 = time.perf_counter()
    inst = cp.Instance(ctx, arrays, mat)
    inst.set_loads(rp, mask, uv)
    rep = inst.solve(allow_not_converged=True, **kw)
    st = inst.state()
    inst.close()
    wall = time.perf_counter() - t0
    out = {"config": CONFIG2, "solver": "FP64 drop-in, Aitken secant, block-Jacobi PCG, adaptive CG rule 2, "
                                         "level predictor (the headline's options)",
           "gpu": {"seconds_e2e": wall, "seconds_device": rep["seconds"], "status": rep["status"],
                   "outer_iters": rep["outer_iters"], "cg_iters": rep["cg_iters"], "levels_done": rep["levels_done"],
                   "rel_err": rep["rel_err"], "kernel_launches": rep["kernel_launches"],
                   "us_per_cg_iter": 1e6 * rep["seconds"] / max(1, rep["cg_iters"]),
                   "yielded": int((np.asarray(st["psi"]) > 1.0 + 1e-12).sum())}}
    if cpu:
        import tempfile

        import oracle

        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import meshgen

        if not os.path.exists(oracle.REF_BIN_CSR):
            out["cpu_prefix"] = {"unavailable": "oracle/_ref/cpref_csr not built"}
            return out
        m = meshgen.hole_plate(-100.0, 100.0, -100.0, 100.0, 20.0, 256, 256, rad_n=1024)
        threads = os.cpu_count()
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "m.bin")
            oracle.write_mesh(path, m["node_xy"], elem4=m["elem4"], borders=m["borders"])
            lines = ["mode phases_csr", f"mesh file {path}", "levels 20", f"cg_eps {cpu_cg_eps}", "outer_eps 1e-6",
                     "max_outer 100000", "prefix_outer 1", "diagram hollomon 210000 250 0.002 0.2",
                     "material 210000 0.3 1", "force 2 0 220 0", "fixborderhor 0", "fixpoint -100 -100"]
            t1 = time.perf_counter()
            r = oracle.run_reference(lines, threads=threads, binary=oracle.REF_BIN_CSR)
            cwall = time.perf_counter() - t1
        cg_it = int(r["cg_per_level"].sum())
        per_it = float(r["cg_seconds"][0]) / max(1, cg_it)
        per_outer = float(r["assembly_seconds"][0] + r["update_seconds"][0])
        est = float(r["setup_seconds"][0]) + per_outer * rep["outer_iters"] + per_it * rep["cg_iters"]
        out["cpu_prefix"] = {"kind": "reference (CSR-direct composition)", "cores": threads,
                             "sample": f"first outer step of increment 1, CG {cpu_cg_eps:g} from zero, "
                                       f"{cg_it} CG iterations", "wall_s": cwall,
                             "setup_s": float(r["setup_seconds"][0]), "assembly_s": float(r["assembly_seconds"][0]),
                             "update_s": float(r["update_seconds"][0]), "cg_s": float(r["cg_seconds"][0]),
                             "ms_per_cg_iter": 1e3 * per_it,
                             "estimated_full_solve_s_at_gpu_iteration_counts": est,
                             "gpu_speedup_vs_estimate": est / wall}
    return out


def fifo_latencies(arrivals, service):
    """Latencies of requests served one at a time in arrival order by a
    single server whose service times are `service` (the plain drop-in):
    start = max(arrival, previous finish)."""
    fin, lat = 0.0, []
    for a, s in zip(arrivals, service):
        fin = max(a, fin) + s
        lat.append(fin - a)
    return lat, fin


STREAMS = {"served": dict(seed=20270101, dof_min=2000, dof_max=500000, increments=(5, 30),
                         text="served stream (DOF log-uniform [2k, 500k], 5-30 load increments)"),
           "batch": dict(seed=20261203, dof_min=2000, dof_max=200000, increments=None,
                         text="batch stream (DOF log-uniform [2k, 200k], one load level)")}


def served_vs_plain_leg(ctx, n_requests, stream="served", rates=(10.0, 100.0, 1000.0), budget_s=120.0,
                        forms=("fp64_lanes", "mixed_batch"), deadline_factor=1.5, lanes=8, **tol):
    """The served-vs-plain comparison on the same requests.

    Requests: the first n of a seeded request stream (STREAMS: the served
    stream, DOF log-uniform in [2k, 500k] and 5-30 load increments, or the
    batch stream, DOF in [2k, 200k] and one level; plates and rings,
    5-segment diagrams).
    plain: each request end to end through the public API, one at a time,
        FP64 drop-in (create the instance from host arrays, loads H2D, solve,
        every result field D2H, destroy); stops taking new requests once
        budget_s is spent, and the served forms then run the same prefix.
    served: the solve service (cp_server) under Poisson arrivals at each rate
        (seeded), host buffers in and every field out; FP64 requests on its
        lanes, mixed-precision requests in its continuous batch. Each run
        ends at deadline_factor x the plain total after the first arrival;
        requests still running then are censored (counted in the latency
        percentiles at the deadline, not in the throughput). Latency =
        submission to completion (the service's clock); throughput =
        completed requests / (last completion - first arrival).
    The plain drop-in's latencies at the same arrivals follow from its
    measured service times (one server, arrival order). Each served result
    is compared with the plain FP64 result of the same request (relative L2
    of u, sigma_i, eps_p_i; the largest over the completed requests)."""
    import random

    import numpy as np

    import cudaplasticity_b200 as cp
    from cudaplasticity_b200 import workload

    kw = dict(FP64_SERVE_KW, **tol)
    st_ = STREAMS[stream]
    seed = st_["seed"]
    reqs, plain = [], []
    t_used = 0.0
    for i in range(n_requests):
        if t_used >= budget_s:
            break
        w = workload.instance(i, seed=seed, dof_min=st_["dof_min"], dof_max=st_["dof_max"],
                              increments=st_["increments"])
        t0 = time.perf_counter()
        inst = cp.Instance(ctx, w["mesh"], w["material"])
        inst.set_loads(w["rp"], w["mask"], w["uv"])
        rep = inst.solve(allow_not_converged=True, precision=cp.CP_PREC_FP64, levels=w["levels"], **kw)
        st = inst.state()
        inst.close()
        dt = time.perf_counter() - t0
        t_used += dt
        reqs.append(w)
        plain.append({"seconds": dt, "status": rep["status"], "outer": rep["outer_iters"], "cg": rep["cg_iters"],
                      "state": st})
        print(json.dumps({"plain": i, "dof": w["params"]["dof"], "levels": w["levels"], "seconds": round(dt, 3),
                          "status": rep["status"], "outer": rep["outer_iters"], "cg": rep["cg_iters"]}),
              file=sys.stderr, flush=True)
    n = len(reqs)
    service = [p["seconds"] for p in plain]
    out = {"workload": "first %d requests of the %s, base seed %d; CG %g, outer %g, outer cap %d, recycled "
                       "initial guesses %d (both arms); FP64 reference = the plain drop-in's result"
                       % (n, st_["text"], seed, kw["cg_tol"], kw["outer_tol"], kw["max_outer"],
                          kw.get("recycle", 0)),
           "requests": n, "dof": [w["params"]["dof"] for w in reqs], "levels": [w["levels"] for w in reqs],
           "plain_fp64_dropin": {"seconds_total": sum(service), "solves_per_s": n / sum(service),
                                 "statuses": sorted({p["status"] for p in plain}),
                                 "outer_iters": [p["outer"] for p in plain], "cg_iters": [p["cg"] for p in plain],
                                 "seconds": service},
           "rates": {}}

    def rel(a, b):
        nb = np.linalg.norm(b)
        return float(np.linalg.norm(a - b) / nb) if nb > 0 else 0.0

    deadline = deadline_factor * sum(service)
    for rate in rates:
        rng = random.Random(seed * 1000 + int(rate))
        arrivals, t = [], 0.0
        for _ in range(n):
            t += rng.expovariate(rate)
            arrivals.append(t)
        p_lat, p_fin = fifo_latencies(arrivals, service)
        plain_sps = n / (p_fin - arrivals[0])
        row = {"plain_fp64_dropin": {"solves_per_s": plain_sps, "p50_s": float(np.percentile(p_lat, 50)),
                                     "p99_s": float(np.percentile(p_lat, 99))}}
        for form in forms:
            srv = cp.Server(fp64_lanes=lanes)
            if form == "fp64_lanes":
                skw = dict(kw, precision=cp.CP_PREC_FP64)
            elif form == "fp64_lanes_mg":  # the lanes with the multigrid-preconditioned CG
                skw = dict(kw, precision=cp.CP_PREC_FP64, precond=2)
            else:
                skw = dict(BATCH_KW, **tol)
            t0 = time.perf_counter()
            rids = []
            for w, a in zip(reqs, arrivals):
                now = time.perf_counter() - t0
                if a > now:
                    time.sleep(a - now)
                rids.append(srv.submit(w["mesh"], w["material"], w["rp"], w["mask"], w["uv"], levels=w["levels"],
                                       **skw))
            lat, errs, statuses, last = {}, {"uv": 0.0, "sig_i": 0.0, "eps_p_i": 0.0}, set(), 0.0
            pending = dict(enumerate(rids))
            while pending and time.perf_counter() - t0 < arrivals[0] + deadline:
                for k, rid in list(pending.items()):
                    try:
                        inst, rep, latency = srv.wait(rid, timeout=0.0)
                    except cp.CuplastError as e:
                        if e.status == cp._capi.CP_ERR_BUSY:
                            continue
                        raise
                    st = inst.state()
                    inst.close()
                    last = max(last, time.perf_counter() - t0)
                    lat[k] = latency
                    statuses.add(rep["status"])
                    for f in errs:
                        errs[f] = max(errs[f], rel(st[f], plain[k]["state"][f]))
                    del pending[k]
                time.sleep(0.01)
            t_end = time.perf_counter() - t0
            srv.close()  # cancels what is still running
            done = len(lat)
            all_lat = [lat[k] if k in lat else t_end - arrivals[k] for k in range(n)]
            sps = done / (last - arrivals[0]) if done and last > arrivals[0] else 0.0
            row[form] = {"solves_per_s": sps, "completed": done, "censored": n - done,
                         "p50_s": float(np.percentile(all_lat, 50)), "p99_s": float(np.percentile(all_lat, 99)),
                         "statuses": sorted(statuses), "max_rel_err_vs_plain_fp64": errs,
                         "within_1e-8": bool(done == n and max(errs.values()) <= 1e-8),
                         "speedup_vs_plain": sps / plain_sps}
            print(json.dumps({"served_vs_plain_rate": rate, "form": form, **row[form]}), file=sys.stderr,
                  flush=True)
        out["rates"][str(int(rate))] = row
    return out


def sharded_service_leg(device, rank, world, dist, n_requests=24, stream="batch", lanes=8, max_outer=300):
    """Instance sharding across GPUs: the first n requests of a seeded stream
    split over the ranks (longest-processing-time first on DOF x increments,
    cudaplasticity_b200.shard), each rank solving its share as one burst
    through the solve service's FP64 lanes on its own GPU; no collective on
    the data path, the per-request records meet on the host (object
    all-gather). Every rank runs it (collectives in the same order);
    throughput = requests / the slowest rank's span. The checksums (sum |u|
    per request) are those of the same requests solved on one GPU: the
    kernels' reductions run in a fixed order."""
    import numpy as np

    import cudaplasticity_b200 as cp
    from cudaplasticity_b200 import shard, workload

    st_ = STREAMS[stream]
    kw = dict(FP64_SERVE_KW, max_outer=max_outer, precision=cp.CP_PREC_FP64)
    # every rank takes the barrier and the all-gather whatever fails locally,
    # so that no rank waits on a collective that another rank skipped
    err, recs, srv, parts = None, {}, None, None
    try:
        reqs = [workload.instance(i, seed=st_["seed"], dof_min=st_["dof_min"], dof_max=st_["dof_max"],
                                  increments=st_["increments"]) for i in range(n_requests)]
        costs = [shard.request_cost(w["params"]["dof"], w["levels"]) for w in reqs]
        parts = shard.partition(costs, world)
        srv = cp.Server(device=device, fp64_lanes=lanes)
    except Exception as exc:  # noqa: BLE001
        err = repr(exc)

    def submit(w):
        return srv.submit(w["mesh"], w["material"], w["rp"], w["mask"], w["uv"], levels=w["levels"], **kw)

    def wait(rid):
        inst, rep, lat = srv.wait(rid, timeout=-1.0)
        u = inst.field("uv")
        inst.close()
        return {"status": rep["status"], "outer": rep["outer_iters"], "cg": rep["cg_iters"], "latency": lat,
                "checksum": float(np.abs(u).sum()), "rank": rank}

    if dist is not None:
        dist.barrier()
    if err is None:
        try:
            recs = shard.run_share(parts[rank], lambda i: reqs[i], submit, wait)
        except Exception as exc:  # noqa: BLE001
            err = repr(exc)
    if srv is not None:
        srv.close()
    got = shard.gather_objects({"records": recs, "error": err}, dist)
    errors = [f"rank {r}: {g['error']}" for r, g in enumerate(got) if g["error"]]
    if errors:
        return {"error": "; ".join(errors)}
    merged = shard.merge_records([g["records"] for g in got])
    out = shard.summarize(merged, n_requests, world)
    out.update(workload="first %d requests of the %s as one burst; FP64 lanes (%d per GPU), CG %g, outer %g, outer "
                        "cap %d" % (n_requests, st_["text"], lanes, kw["cg_tol"], kw["outer_tol"], max_outer),
               split="longest-processing-time first on DOF x increments",
               shares=[{"rank": r, "requests": parts[r], "seconds": max((merged[i]["done_at"] for i in parts[r]),
                                                                         default=0.0)} for r in range(world)],
               checksums=[merged[i]["checksum"] for i in range(n_requests)])
    return out


def run_sharded(args):
    """bench.py --sharded N [under torchrun]: the sharded-service leg alone."""
    import cudaplasticity_b200 as cp  # noqa: F401  (loads the library before the process group)

    rank, world, local = dist_env()
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist_mod

        torch.cuda.set_device(local)
        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = dist_mod
    out = sharded_service_leg(local, rank, world, dist, n_requests=args.sharded)
    if rank == 0:
        print(json.dumps({"sharded_service": out}), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_product_arm(args):
    import numpy as np

    import cudaplasticity_b200 as cp
    from cudaplasticity_b200.ranks import max_over_ranks, replica_throughput

    rank, world, local = dist_env()
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist_mod

        torch.cuda.set_device(local)
        dist_mod.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
        dist = dist_mod
    device = local
    ctx = cp.Context(device)
    mesh, arrays, mat, rp, mask, uv = build_problem()

    # resident arm: instance built once, every step = reset + full solve
    inst = cp.Instance(ctx, arrays, mat)
    inst.set_loads(rp, mask, uv)

    def one_solve():
        inst.reset_state()
        inst.set_loads(rp, mask, uv)
        return inst.solve(**SOLVE_KW)

    for _ in range(args.warmup):
        one_solve()

    def barrier():
        if dist is not None:
            dist.barrier()

    times, reps = [], []
    with ClockSampler(device) as clocks:
        barrier()
        for _ in range(args.steps):
            flush_l2(device)
            rep = one_solve()
            times.append(rep["seconds"])
            reps.append(rep)
        barrier()
    total = max_over_ranks(sum(times), dist, device)
    value = replica_throughput(world, len(times), total)

    # end to end through the public C ABI with host buffers: mesh upload and
    # set-up, loads H2D, solve, every result field D2H, teardown
    e2e_times = []
    h2d = arrays["node_xy"].nbytes + arrays["elem4"].nbytes + rp.nbytes + mask.nbytes + uv.nbytes
    d2h = 0
    for k in range(max(1, min(args.steps, 3)) + 1):
        t0 = time.perf_counter()
        e = cp.Instance(ctx, arrays, mat)
        e.set_loads(rp, mask, uv)
        e.solve(**SOLVE_KW)
        st = e.state()
        e.close()
        dt = time.perf_counter() - t0
        d2h = sum(v.nbytes for v in st.values())
        if k > 0:
            e2e_times.append(dt)
    e2e_total = max_over_ranks(sum(e2e_times), dist, device)
    e2e_value = replica_throughput(world, len(e2e_times), e2e_total)

    # accuracy of the timed configuration against a tight FP64 solve
    state = inst.state()
    inst.reset_state()
    inst.set_loads(rp, mask, uv)
    inst.solve(cg_tol=1e-13, outer_tol=1e-12, max_outer=5000, levels=10, aitken=1, adaptive_cg=1, precond=1,
               max_cg=5_000_000)
    tight = inst.state()

    def rel(k):
        return float(np.linalg.norm(state[k] - tight[k]) / np.linalg.norm(tight[k]))

    accuracy = {k: rel(k) for k in ("uv", "sig_i", "eps_p_i")}

    # configuration 3: the same job in mixed precision (FP32 values and inner
    # CG inside FP64 defect correction, FP64 u, sums and secant update),
    # under the timed tolerances and under tight ones, each against the tight
    # FP64 state
    def mixed_solve(**kw):
        inst.reset_state()
        inst.set_loads(rp, mask, uv)
        r3 = inst.solve(precision=cp.CP_PREC_MIXED, inner_tol=1e-3, **kw)
        st3 = inst.state()
        return r3, {k: float(np.linalg.norm(st3[k] - tight[k]) / np.linalg.norm(tight[k]))
                    for k in ("uv", "sig_i", "eps_p_i")}

    try:
        r3, e3 = mixed_solve(**dict(SOLVE_KW, adaptive_cg=1))
        r3t, e3t = mixed_solve(cg_tol=1e-12, outer_tol=1e-10, max_outer=5000, levels=10, aitken=1, adaptive_cg=1,
                               precond=1, max_cg=5_000_000)
        config3 = {"workload": "configuration-1 job in mixed precision (FP32 K values and inner CG, FP64 defect "
                               "correction, u, dot-product sums and secant update)",
                   "timed_tolerances": {"solves_per_s": 1.0 / r3["seconds"], "outer_iters": r3["outer_iters"],
                                        "cg_iters": r3["cg_iters"], "fp64_residuals": r3["fp64_spmv"],
                                        "rel_l2_vs_tight_fp64": e3},
                   "tight_tolerances": {"cg_tol": 1e-12, "outer_tol": 1e-10, "seconds": r3t["seconds"],
                                        "rel_l2_vs_tight_fp64": e3t, "within_1e-8": max(e3t.values()) <= 1e-8}}
    except cp.CuplastError as exc:  # an auxiliary figure: report the failure, keep the line
        config3 = {"error": str(exc)}

    # roofline of the dominant kernel (the SpMV P of the CG), live CUDA events:
    # on this workload, and on the 2.1M-DOF 1024x1024 O-grid plate ("CG GB/s")
    peak, peak_kind = measured_peak_hbm()
    import ctypes

    def bench_cg(instance, precision, precond, iters):
        mp, mu, bp, bu = (ctypes.c_double() for _ in range(4))
        instance.ctx.check(cp._capi.lib().cp_bench_cg(instance._h, precision, precond, iters, ctypes.byref(mp),
                                                      ctypes.byref(mu), ctypes.byref(bp), ctypes.byref(bu)))
        return mp.value, mu.value, bp.value, bu.value

    def bench_mg(instance, iters):
        """Per-part timings of the multigrid PCG (cp_bench_mg): P, U, R0, the
        coarse levels, S0 per iteration and the per-outer-iteration set-up."""
        ms, by = (ctypes.c_double * 6)(), (ctypes.c_double * 6)()
        instance.ctx.check(cp._capi.lib().cp_bench_mg(instance._h, iters, ms, by))
        names = ["P", "U", "R0", "coarse", "S0", "setup"]
        return {k: {"ms": ms[i], "bytes": by[i], "gbs": by[i] / (ms[i] * 1e-3) / 1e9,
                    "frac": by[i] / (ms[i] * 1e-3) / 1e9 / peak} for i, k in enumerate(names)}

    # this workload's own CG: each linear solve is one k_c_solve launch (the
    # whole CG inside one thread-block cluster, matrix and records in shared
    # memory). Time per CG iteration from one elastic PCG solve from zero
    # (CUDA events of cp_solve around assembly + solve + update; the solve
    # dominates), against the algorithmic bytes of one CG iteration
    # nnz (8 + 4) + 4 (N + 1) + 2 N 8 + 9 N 8 (N = DOF).
    def small_cg_roofline():
        n_nodes, _, nnz, _ = inst.sizes()
        ndof = 2 * n_nodes
        b_iter = nnz * 12 + 4 * (ndof + 1) + 2 * ndof * 8 + 9 * ndof * 8
        t_iter = None
        for _ in range(3):
            inst.reset_state()
            inst.set_loads(rp, mask, uv)
            r1 = inst.solve(cg_tol=1e-10, outer_tol=1e300, max_outer=1, levels=1, precond=1, max_cg=2_000_000)
            t = r1["seconds"] / max(1, r1["cg_iters"])
            t_iter = t if t_iter is None else min(t_iter, t)
        return b_iter, t_iter

    try:
        b_iter, t_iter = small_cg_roofline()
    except cp.CuplastError as exc:  # an auxiliary figure: report the failure, keep the line
        b_iter, t_iter = None, None
        small_error = str(exc)
    if t_iter is None:
        roof_small = {"kernel": "k_c_solve", "error": small_error}
    else:
        roof_small = {"bound": "hbm", "kernel": "k_c_solve (FP64 PCG in one thread-block cluster, per CG iteration)",
                      "achieved": b_iter / t_iter / 1e9, "peak": peak, "unit": "GB/s",
                      "frac": b_iter / t_iter / 1e9 / peak, "traffic": None, "bytes_per_launch": b_iter,
                      "ms_per_launch": t_iter * 1e3, "peak_kind": peak_kind,
                      "note": "per CG iteration of the 8320-DOF instance; its matrix and vectors live in shared "
                              "memory and registers, so HBM does not bind: the iteration is latency-bound"}
    inst.close()
    big = cp.Mesh.rect_with_hole(-100.0, 100.0, -100.0, 100.0, 20.0, 256, 256, rad_n=1024)
    L = cp.Loads().set_force(2, 0.0, 220.0).fix_border_hor(0).fix_point(-100.0, -100.0)
    brp, bmask, buv = L.build(big)
    binst = cp.Instance(ctx, big.arrays(), mat)
    binst.set_loads(brp, bmask, buv)
    rows = {}
    for prec, name in ((cp.CP_PREC_FP64, "fp64"), (cp.CP_PREC_MIXED, "fp32")):
        binst.set_field("uv", np.zeros_like(brp))
        rows[name] = bench_cg(binst, prec, 0, 100)
    # the FP64 CG iteration that instances too large for one cluster run
    # (configuration 2): one k_f_iter launch per block-Jacobi PCG iteration
    binst.set_field("uv", np.zeros_like(brp))
    fms, fby = ctypes.c_double(), ctypes.c_double()
    binst.ctx.check(cp._capi.lib().cp_bench_cg_fused(binst._h, 1, 200, ctypes.byref(fms), ctypes.byref(fby)))
    # elements assembled per second (fillGlobalStiffness on the 1,048,576-element
    # mesh, CUDA events around the launches) and DOF-iterations per second
    throughput = {"assembly_mesh": "1024x1024 O-grid plate, 1,048,576 Q4, FP64 values"}
    try:
        ams, aby = ctypes.c_double(), ctypes.c_double()
        binst.ctx.check(cp._capi.lib().cp_bench_assemble(binst._h, cp.CP_PREC_FP64, 10, ctypes.byref(ams),
                                                          ctypes.byref(aby)))
        big_nodes, big_elems = binst.sizes()[:2]
        throughput.update(elements_assembled_per_s=big_elems / (ams.value * 1e-3), assembly_ms=ams.value,
                          assembly_gbs=aby.value / (ams.value * 1e-3) / 1e9, assembly_bytes=aby.value)
    except cp.CuplastError as exc:  # an auxiliary figure: report the failure, keep the line
        big_nodes = binst.sizes()[0]
        throughput["assembly_error"] = str(exc)
    mg_parts = None
    if SOLVE_KW["precond"] == 2:
        try:
            binst.set_field("uv", np.zeros_like(brp))
            mg_parts = {"plate_2.1M_dof": bench_mg(binst, 20)}
        except cp.CuplastError as exc:  # an auxiliary figure: report the failure, keep the line
            mg_parts = {"error": str(exc)}
    binst.close()
    mp, mu, bp, bu = rows["fp64"]
    throughput["dof_iterations_per_s_2M"] = 2 * big_nodes / ((mp + mu) * 1e-3)
    cg_large = {k: {"spmv_gbs": b / (m * 1e-3) / 1e9, "update_gbs": c / (n * 1e-3) / 1e9, "ms_spmv": m,
                    "ms_update": n, "us_per_cg_iter": 1e3 * (m + n)} for k, (m, n, b, c) in rows.items()}
    # "CG GB/s": the FP64 CG iteration of the 2.1M-DOF plate (k_f_iter, the
    # kernel that takes 90 % of a configuration-2 solve), live CUDA events
    roofline = {"bound": "hbm", "kernel": "k_f_iter (FP64 block-Jacobi PCG iteration, one launch) on the 2.1M-DOF "
                                          "1024x1024 O-grid plate",
                "achieved": fby.value / (fms.value * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                "frac": fby.value / (fms.value * 1e-3) / 1e9 / peak, "traffic": 622.5e6,
                "traffic_note": "dram__bytes_read.sum + dram__bytes_write.sum of one k_f_iter launch on this mesh "
                                "(ncu capture, profiles/k_f_iter_2M.md)",
                "bytes_per_launch": fby.value, "ms_per_launch": fms.value, "peak_kind": peak_kind,
                "why_this_kernel": "the metric's CG GB/s: the dominant kernel of the configuration-2 solve "
                                   "(k_f_iter, 114 us x 924k iterations of its 105 s); the headline step's own "
                                   "kernel, k_c_solve, keeps the instance on chip and is latency-bound, so its "
                                   "HBM fraction is reported apart as roofline_headline"}
    mp32, mu32, bp32, bu32 = rows["fp32"]
    roof_fp32 = {"bound": "hbm", "kernel": "k_cg_p<float> (mixed precision SpMV + direction) on the 2.1M-DOF plate",
                 "achieved": bp32 / (mp32 * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                 "frac": bp32 / (mp32 * 1e-3) / 1e9 / peak, "traffic": None, "bytes_per_launch": bp32,
                 "ms_per_launch": mp32, "peak_kind": peak_kind}

    cpu = err_ref = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        c = cpu_baseline_run()
        cpu = {"value": 1.0 / c["seconds"], "unit": "solves/s", "cores": c["cores"], "kind": c["kind"],
               "sample": "one full 8320-DOF hole-plate solve (10 levels, CG 1e-10, outer 1e-6), reference CPU path "
                         f"through its phase functions, {c['outer']} outer / {c['cg']} CG iterations"}
        err_ref = error_vs_reference(state, c["state"], tight)

    batched = served = roof_batched = config2 = None
    def aux(name, fn):
        """An auxiliary leg: its failure is reported in the line, which is still printed."""
        try:
            return fn()
        except Exception as exc:  # noqa: BLE001
            print(json.dumps({"leg_failed": name, "error": repr(exc)}), file=sys.stderr, flush=True)
            return {"error": repr(exc)}

    sharded = None
    if world > 1 and not args.skip_served:
        # every rank: its share of the batch-stream requests on its own GPU
        try:
            sharded = sharded_service_leg(device, rank, world, dist, n_requests=args.serve_requests)
        except Exception as exc:  # noqa: BLE001
            sharded = {"error": repr(exc)}
    # the single-GPU comparisons (N = 1 figures; with N > 1 the ranks have
    # left after the sharded leg)
    if rank == 0 and world == 1 and not args.skip_served:
        # the metric: the same requests served and one at a time through the
        # plain FP64 drop-in, at three Poisson rates
        served = aux("served_vs_plain", lambda: served_vs_plain_leg(
            ctx, args.serve_requests, stream="batch", budget_s=args.serve_budget, forms=("fp64_lanes",),
            max_outer=300))
    if rank == 0 and world == 1 and not args.skip_batched:
        batched = aux("batched", lambda: batched_leg(ctx, window_s=args.batched_window))
        roof_batched = aux("roofline_batched", lambda: cg_kernel_roofline(ctx))
    if rank == 0 and world == 1 and not args.skip_config2:
        config2 = aux("config2", lambda: config2_leg(ctx, cpu=not args.skip_cpu, cpu_cg_eps=0.1))

    launches = sum(r["kernel_launches"] for r in reps)
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": line_config(world),
            "solver": f"FP64, Aitken secant, {PRECOND_NAMES[SOLVE_KW['precond']]}, adaptive CG tolerance "
                      "max(1e-10, 0.2 relErr) until relErr <= 1e-6, then 1e-10; levels from the "
                      "third on start from the linear extrapolation of the last two"
                      + ("; each linear solve starts from the Galerkin projection onto the level's last "
                         f"{SOLVE_KW['recycle']} solution increments" if SOLVE_KW["recycle"] else ""),
            "cg_form": ("graph loop: P, U, then the V-cycle (restrict per level, dense coarsest "
                        "inverse, prolongation fused into post-smoothing), one kernel each"
                        if SOLVE_KW["precond"] == 2 else os.environ.get("CUPLAST_FP64_CG") or
                        "one thread-block cluster per linear solve (on chip) where the instance fits"),
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": int(launches), "roofline": roofline, "roofline_headline": roof_small,
            "roofline_fp32_spmv": roof_fp32,
            "cg_large_mesh": cg_large, "config3": dict(config3, spmv_gbs_2M={k: v["spmv_gbs"] for k, v in
                                                                         cg_large.items()}),
            "multigrid_parts": mg_parts, "cpu_baseline": cpu, "clocks": clocks.summary(),
            "accuracy_vs_tight_fp64": accuracy, "error_vs_reference": err_ref, "batched": batched,
            "roofline_batched": roof_batched, "served_vs_plain": served, "config2": config2,
            "sharded_service": sharded,
            "throughput": dict(throughput, dof_iterations_per_s_headline=2 * arrays["node_xy"].shape[0] *
                               sum(r["cg_iters"] for r in reps) / sum(times)),
            "detail": {"outer_iters": reps[-1]["outer_iters"], "cg_iters": reps[-1]["cg_iters"],
                       "step_seconds": times}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


CG_ONLY_KW = dict(cg_tol=1e-12, outer_tol=1e-9, max_outer=50, max_cg=5_000_000, precond=1, aitken=1, adaptive_cg=0,
                  inner_tol=1e-3)


def cg_kernel_roofline(ctx, n=512, warm_trips=3, trips=10, seed=20261203):
    """Live roofline of the batched CG iteration kernel (k_batch_cg, ITER
    phase): n resident batch-stream instances with tight, non-adaptive linear
    solves, so every launch after the warm-up is a CG iteration of every
    instance; CUDA-event time per iteration of the whole batch and the
    algorithmic bytes one iteration must move."""
    import cudaplasticity_b200 as cp
    from cudaplasticity_b200 import workload

    insts = []
    for i in range(n):
        w = workload.instance(i, seed=seed)
        inst = cp.Instance(ctx, w["mesh"], w["material"])
        inst.set_loads(w["rp"], w["mask"], w["uv"])
        insts.append(inst)
    b = cp.Batch(ctx, max_instances=n)
    for inst in insts:
        b.add(inst, levels=1, **CG_ONLY_KW)
    b.run(max_trips=warm_trips)
    b.autotune()
    cg0 = [b.progress(s)[2]["cg_iters"] for s in range(n)]
    b.run(max_trips=trips)
    sec = b.last_run_ms() * 1e-3  # CUDA events around the run on the batch's stream
    done_iters = [b.progress(s)[2]["cg_iters"] - cg0[s] for s in range(n)]
    phases = [b.progress(s)[0] for s in range(n)]
    # per 2x2 block: 4 FP32 values + one column; per node: read the 32-byte
    # record, p, w, kp, r (FP32 pairs), x (FP64 pair), mask, block-Jacobi
    # inverse; write p, kp, x, r, w and the new record
    per_iter = []
    nodes = 0
    for inst in insts:
        nn, ne, nnz, nadj = inst.sizes()
        per_iter.append(20.0 * (nnz // 4) + 178.0 * nn)
        nodes += nn
    b.close()
    for inst in insts:
        inst.close()
    moved = sum(k * bi for k, bi in zip(done_iters, per_iter))
    iters = max(done_iters)  # launches of the iteration kernel that did work
    bytes_iter = moved / iters
    peak, peak_kind = measured_peak_hbm()
    us = 1e6 * sec / iters
    gbs = moved / sec / 1e9
    return {"bound": "hbm", "kernel": "k_batch_cg (CG iteration of %d resident instances, %d DOF)" % (n, 2 * nodes),
            "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak, "traffic": None,
            "bytes_per_launch": bytes_iter, "ms_per_launch": us * 1e-3, "peak_kind": peak_kind,
            "iterations_timed": iters, "instance_iterations": int(sum(done_iters)),
            "in_cg_at_end": phases.count(5)}


def batched_probe(n, trips):
    """A fixed slice of batched CG work for profilers: n resident batch-stream
    instances with tight, non-adaptive linear solves (every launch after the
    first trips is a CG iteration), `trips` graph trips; prints the time."""
    import cudaplasticity_b200 as cp
    from cudaplasticity_b200 import workload

    ctx = cp.Context(0)
    insts = []
    for i in range(n):
        w = workload.instance(i)
        inst = cp.Instance(ctx, w["mesh"], w["material"])
        inst.set_loads(w["rp"], w["mask"], w["uv"])
        insts.append(inst)
    b = cp.Batch(ctx, max_instances=n)
    for inst in insts:
        b.add(inst, levels=1, **CG_ONLY_KW)
    b.run(max_trips=3)
    ms = b.autotune()
    t0 = time.perf_counter()
    b.run(max_trips=trips)
    dt = time.perf_counter() - t0
    print(json.dumps({"batched_probe": n, "trips": trips, "ms_per_trip": 1e3 * dt / trips, "stats": b.stats(),
                      "autotune_ms_per_sweep": ms, "tiles": [b.tile(k) for k in range(4, 14)]}))
    b.close()
    for inst in insts:
        inst.close()
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--skip-cpu", action="store_true", help="omit the CPU-baseline leg")
    ap.add_argument("--skip-batched", action="store_true", help="omit the batched (batch stream, DOF 2k-200k) leg")
    ap.add_argument("--skip-served", action="store_true", help="omit the served (served stream, DOF 2k-500k) leg")
    ap.add_argument("--batched-window", type=float, default=20.0, help="seconds counted in the saturation run")
    ap.add_argument("--compare", type=int, metavar="N",
                    help="like-for-like run only: the first N batch-stream requests, plain FP64 one at a time vs batched")
    ap.add_argument("--compare-max-outer", type=int, default=100)
    ap.add_argument("--serve-requests", type=int, default=24, help="requests in the served-vs-plain leg")
    ap.add_argument("--serve-budget", type=float, default=60.0,
                    help="seconds of plain solves after which the served-vs-plain sample stops growing")
    ap.add_argument("--skip-config2", action="store_true", help="omit the configuration-2 leg")
    ap.add_argument("--batched-probe", type=int, nargs=2, metavar=("N", "TRIPS"),
                    help="profiling aid: N resident batch-stream instances, TRIPS graph trips, then exit")
    ap.add_argument("--config2", action="store_true",
                    help="configuration 2 only (2.1M-DOF Hollomon plate, 20 increments) and its CPU prefix, then exit")
    ap.add_argument("--svp", type=int, metavar="N",
                    help="served-vs-plain leg only: the first N requests of --svp-stream, then exit")
    ap.add_argument("--svp-stream", default="served", choices=sorted(STREAMS))
    ap.add_argument("--svp-budget", type=float, default=120.0, help="seconds of plain solves before the prefix stops")
    ap.add_argument("--svp-outer-tol", type=float, default=1e-6)
    ap.add_argument("--svp-cg-tol", type=float, default=1e-10)
    ap.add_argument("--svp-max-outer", type=int, default=2000, help="outer-iteration cap per load level, both arms")
    ap.add_argument("--svp-forms", default="fp64_lanes,mixed_batch")
    ap.add_argument("--svp-rates", default="10,100,1000", help="Poisson arrival rates (requests/s), comma-separated")
    ap.add_argument("--svp-lanes", type=int, default=8, help="FP64 lanes of the solve service")
    ap.add_argument("--sharded", type=int, metavar="N",
                    help="sharded-service leg only (the first N batch-stream requests split over the ranks), then exit")
    ap.add_argument("--recycle", type=int, default=SOLVE_KW["recycle"], choices=range(0, 7),
                    help="initial guesses from the last N solution increments of a load level (0: off)")
    ap.add_argument("--precond", type=int, default=SOLVE_KW["precond"], choices=[0, 1, 2],
                    help="linear solver of the headline and of the FP64 served arm: 0 CG, 1 block-Jacobi PCG, "
                         "2 multigrid PCG")
    args = ap.parse_args()
    SOLVE_KW["precond"] = args.precond
    SOLVE_KW["recycle"] = args.recycle
    FP64_SERVE_KW["recycle"] = args.recycle
    FP64_SERVE_KW["precond"] = args.precond
    if args.batched_probe:
        batched_probe(*args.batched_probe)
        return
    if args.config2:
        import cudaplasticity_b200 as cp

        ctx = cp.Context(0)
        print(json.dumps({"config2": config2_leg(ctx, cpu=not args.skip_cpu)}), flush=True)
        ctx.close()
        return
    if args.sharded:
        run_sharded(args)
        return
    if args.svp:
        import cudaplasticity_b200 as cp

        ctx = cp.Context(0)
        print(json.dumps({"served_vs_plain": served_vs_plain_leg(
            ctx, args.svp, stream=args.svp_stream, budget_s=args.svp_budget, forms=tuple(args.svp_forms.split(",")),
            rates=tuple(float(x) for x in args.svp_rates.split(",")), lanes=args.svp_lanes,
            outer_tol=args.svp_outer_tol, cg_tol=args.svp_cg_tol, max_outer=args.svp_max_outer)}), flush=True)
        ctx.close()
        return
    if args.compare:
        import cudaplasticity_b200 as cp

        ctx = cp.Context(0)
        print(json.dumps({"compare": compare_leg(ctx, args.compare, max_outer=args.compare_max_outer)}), flush=True)
        ctx.close()
        return
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_product_arm(args)


if __name__ == "__main__":
    main()
