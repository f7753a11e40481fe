"""Benchmark: converged plastic solves per second on one B200 (per GPU, replicas).

Workload (configuration "plain method, small", the reference's CPU-runnable
case): plane-stress 200 x 200 mm plate with a centred 20 mm hole, O-grid of 64
circumferential x 64 radial quads (4160 nodes, 8320 DOF), E = 210 GPa, nu = 0.3,
bilinear hardening sigma_y = 250 MPa, E_t = 2 GPa; 200 MPa traction on the top
edge in 10 equal increments; bottom edge fixed in y, bottom-left node fixed;
CG tolerance 1e-10, outer (secant) tolerance 1e-6. Quads on the O-grid nodes:
the reference has no triangle element. Synthetic, seeded-free (deterministic).

One step = one complete solve (all 10 load levels to convergence). The product
arm runs the FP64 drop-in path (Aitken-relaxed secant iteration, block-Jacobi
PCG with the linear tolerance following the outer error; same fixed point as
the reference). ``--impl reference`` runs the reference implementation's own
CPU path (oracle/_ref/cpref, built from its sources) on the same job with all
host cores.

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

WORKLOAD = dict(workload="config1_hole_plate_ogrid64x64_q4", plate_mm=200, hole_radius_mm=20, n_circ=64, n_rad=64,
                nodes=4160, dof=8320, elements=4096, E_mpa=210000, nu=0.3, sigma_y=250, E_t=2000, traction_mpa=200,
                increments=10, cg_tol=1e-10, outer_tol=1e-6)
SOLVE_KW = dict(cg_tol=1e-10, outer_tol=1e-6, max_outer=2000, levels=10, aitken=1, adaptive_cg=1, precond=1,
                max_cg=2_000_000)
METRIC = "converged solves/s (config-1 plate, FP64, <=1e-6 outer / 1e-10 CG)"


def build_problem():
    import cudaplasticity_b200 as cp

    mesh = cp.Mesh.rect_with_hole(-100.0, 100.0, -100.0, 100.0, 20.0, 16, 16, rad_n=64)
    loads = cp.Loads().set_force(2, 0.0, 200.0).fix_border_hor(0).fix_point(-100.0, -100.0)
    rp, mask, uv = loads.build(mesh)
    mat = cp.material(210000.0, 0.3, diagram="linear", sigma_t=250.0, k_t=2000.0)
    return mesh, mesh.arrays(), mat, rp, mask, uv


def reference_job_lines(mesh_path):
    return ["mode phases", f"mesh file {mesh_path}", "levels 10", "cg_eps 1e-10", "outer_eps 1e-6",
            "max_outer 100000", "diagram linear 210000 250 2000", "material 210000 0.3 1", "force 2 0 200 0",
            "fixborderhor 0", "fixpoint -100 -100"]


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


def cpu_baseline_run(threads=None):
    """The reference's own CPU path on the same job (oracle/_ref/cpref), or the
    oracle restatement where the reference could not be built."""
    import tempfile

    import oracle

    threads = threads or os.cpu_count()
    mesh, arrays, _, _, _, _ = build_problem()
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "m.bin")
        oracle.write_mesh(path, arrays["node_xy"], elem4=arrays["elem4"], borders=arrays["borders"])
        lines = reference_job_lines(path)
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
        pass  # CPU code: nothing to warm beyond the first call, which is timed like the others
    info = None
    for _ in range(args.steps):
        info = cpu_baseline_run()
        steps.append(info["seconds"])
    total = sum(steps)
    value = len(steps) / total
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(steps),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": WORKLOAD,
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": info["cores"], "kind": info["kind"],
                             "sample": "full config-1 solve (10 levels) per step, reference CPU path, all host cores"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "detail": {"outer_iters": info["outer"], "cg_iters": info["cg"]}}
    print(json.dumps(line), flush=True)


def flush_l2(ctx_dev):
    """Writes 512 MB (4x the 126 MB L2) so the next step starts cold."""
    import torch

    buf = getattr(flush_l2, "buf", None)
    if buf is None:
        buf = flush_l2.buf = torch.empty(64 * 1024 * 1024, dtype=torch.float64, device=f"cuda:{ctx_dev}")
    buf.fill_(1.0)
    torch.cuda.synchronize(ctx_dev)


def run_product_arm(args):
    import numpy as np

    import cudaplasticity_b200 as cp

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
    total = sum(times)
    if dist is not None:
        import torch

        t = torch.tensor([total], dtype=torch.float64, device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total = float(t.item())
    value = world * len(times) / total

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
    e2e_total = sum(e2e_times)
    if dist is not None:
        import torch

        t = torch.tensor([e2e_total], dtype=torch.float64, device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e_value = world * len(e2e_times) / e2e_total

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

    # roofline of the dominant kernel (the SpMV P of the CG), live CUDA events:
    # on this workload, and on the 2.1M-DOF configuration-2 mesh ("CG GB/s")
    peak, peak_kind = measured_peak_hbm()
    import ctypes

    def bench_cg(instance, precision, precond, iters):
        mp, mu, bp, bu = (ctypes.c_double() for _ in range(4))
        instance.ctx.check(cp._capi.lib().cp_bench_cg(instance._h, precision, precond, iters, ctypes.byref(mp),
                                                      ctypes.byref(mu), ctypes.byref(bp), ctypes.byref(bu)))
        return mp.value, mu.value, bp.value, bu.value

    inst.reset_state()
    inst.set_loads(rp, mask, uv)
    mp, mu, bp, bu = bench_cg(inst, cp.CP_PREC_FP64, 1, 200)
    roof_small = {"bound": "hbm", "kernel": "k_cg_p<double,pcg>", "achieved": bp / (mp * 1e-3) / 1e9,
                  "peak": peak, "unit": "GB/s", "frac": bp / (mp * 1e-3) / 1e9 / peak, "traffic": None,
                  "bytes_per_launch": bp, "ms_per_launch": mp, "peak_kind": peak_kind,
                  "note": "8320-DOF instance: 1.8 MB matrix is L2-resident; latency-bound, the HBM roof does not bind"}
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
    binst.close()
    mp, mu, bp, bu = rows["fp64"]
    cg_large = {k: {"spmv_gbs": b / (m * 1e-3) / 1e9, "update_gbs": c / (n * 1e-3) / 1e9, "ms_spmv": m,
                    "ms_update": n, "us_per_cg_iter": 1e3 * (m + n)} for k, (m, n, b, c) in rows.items()}
    roofline = {"bound": "hbm", "kernel": "k_cg_p<double> (SpMV+dot) on the 2.1M-DOF config-2 mesh",
                "achieved": bp / (mp * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                "frac": bp / (mp * 1e-3) / 1e9 / peak, "traffic": 402.7e6,
                "traffic_note": "dram__bytes_read.sum + dram__bytes_write.sum of one k_cg_p<double> launch (ncu capture)",
                "bytes_per_launch": bp, "ms_per_launch": mp, "peak_kind": peak_kind}

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        c = cpu_baseline_run()
        cpu = {"value": 1.0 / c["seconds"], "unit": "solves/s", "cores": c["cores"], "kind": c["kind"],
               "sample": "one full config-1 solve (10 levels, CG 1e-10, outer 1e-6), reference CPU path, "
                         f"{c['outer']} outer / {c['cg']} CG iterations"}

    launches = sum(r["kernel_launches"] for r in reps)
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(WORKLOAD, parallelism=f"replicas x{world}", l2="flushed (512 MB write) between steps",
                           solver="FP64, Aitken secant, block-Jacobi PCG, adaptive CG tolerance"),
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": int(launches), "roofline": roofline, "roofline_this_workload": roof_small,
            "cg_large_mesh": cg_large, "cpu_baseline": cpu, "clocks": clocks.summary(),
            "accuracy_vs_tight_fp64": accuracy,
            "detail": {"outer_iters": reps[-1]["outer_iters"], "cg_iters": reps[-1]["cg_iters"],
                       "step_seconds": times}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--skip-cpu", action="store_true", help="omit the CPU-baseline leg")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_product_arm(args)


if __name__ == "__main__":
    main()
