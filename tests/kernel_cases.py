"""One kernel at a time, on a fixed input, for profilers (ncu -k <kernel>).

    python tests/kernel_cases.py <case> [--repeat R]

Cases (each prints one JSON line with its host-side facts):

* ``assemble``   -- k_assemble on the 1024x1024 O-grid plate (1,048,576 Q4,
  2.1M DOF), R launches (cp_bench_assemble: CUDA events around them);
* ``update``     -- k_update (strain, stress, secant update, exit norm) on the
  same plate, R launches after one linear solve;
* ``cg_cluster`` -- k_c_solve: R block-Jacobi PCG solves of the 64x64 O-grid
  plate (8320 DOF) from zero (with the assembly and the secant update of a
  one-iteration cp_solve around each), the whole solve in one thread-block
  cluster; prints the time per CG iteration;
* ``cg_graph``   -- the same solve with one k_f_iter launch per iteration
  (run with CUPLAST_FP64_CG=fused CUPLAST_NO_GRAPH=1 so that every launch is
  visible to the profiler);
* ``cg_large``   -- k_cg_p / k_cg_u on the 2.1M-DOF plate, R iterations
  (cp_bench_cg), FP64 values or (``--fp32``) the mixed mode's FP32 ones;
* ``cg_fused_large`` -- k_f_iter, the FP64 form of instances too large for one
  cluster: R iterations of one block-Jacobi PCG solve on the 2.1M-DOF plate
  (run with CUPLAST_NO_GRAPH=1 so that every launch is visible);
* ``cg_mg``      -- the multigrid-preconditioned solve (cp_solve_opts.precond
  2: set-up kernels, then k_mg_p / k_mg_u / k_mg_restrict0 /
  k_mg_coarse_cycle / k_mg_smooth0 per iteration) of the 64x64 plate from
  zero, R linear solves;
* ``cg_mg_large`` -- the same on the 2.1M-DOF plate, one linear solve to 1e-6;
* ``mg_parts``   -- cp_bench_mg on the 2.1M-DOF plate: the set-up once, then
  R iterations with CUDA events around P, U, R0, the coarse levels and S0;
  ``mg_parts_small`` the same on the 64x64 plate.

The inputs are the benchmark's (bilinear steel, top traction), built the
same way; nothing here is timed for a report.
"""
import argparse
import ctypes
import json
import sys

import numpy as np

import os

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from cudaplasticity_b200 import CP_PREC_FP64, Context, Instance, Loads, Mesh, material  # noqa: E402
from cudaplasticity_b200 import _capi as C  # noqa: E402


def _plate(n_circ4, rad_n):
    mesh = Mesh.rect_with_hole(-100.0, 100.0, -100.0, 100.0, 20.0, n_circ4, n_circ4, rad_n=rad_n)
    rp, mask, uv = Loads().set_force(2, 0.0, 200.0).fix_border_hor(0).fix_point(-100.0, -100.0).build(mesh)
    mat = material(210000.0, 0.3, diagram="linear", sigma_t=250.0, k_t=2000.0)
    return mesh, mat, rp, mask, uv


def _instance(ctx, n_circ4, rad_n):
    mesh, mat, rp, mask, uv = _plate(n_circ4, rad_n)
    inst = Instance(ctx, mesh.arrays(), mat)
    inst.set_loads(rp, mask, uv)
    return inst


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("case", choices=["assemble", "update", "cg_cluster", "cg_graph", "cg_large", "cg_fused_large",
                                     "cg_mg", "cg_mg_large", "mg_parts", "mg_parts_small"])
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--fp32", action="store_true", help="cg_large: the mixed mode's FP32 values")
    a = ap.parse_args(argv)
    ctx = Context(0)
    out = {"case": a.case}
    if a.case in ("mg_parts", "mg_parts_small"):
        inst = _instance(ctx, 256, 1024) if a.case == "mg_parts" else _instance(ctx, 16, 64)
        ms, by = (ctypes.c_double * 6)(), (ctypes.c_double * 6)()
        inst.set_field("uv", np.zeros(2 * inst.sizes()[0]))
        ctx.check(C.lib().cp_bench_mg(inst._h, a.repeat, ms, by))
        out.update(nodes=inst.sizes()[0], parts=["P", "U", "R0", "coarse", "S0", "setup"], ms=list(ms),
                   bytes=list(by))
        inst.close()
    elif a.case in ("cg_mg", "cg_mg_large"):
        inst = _instance(ctx, 16, 64) if a.case == "cg_mg" else _instance(ctx, 256, 1024)
        n_nodes = inst.sizes()[0]
        reps = []
        for _ in range(a.repeat if a.case == "cg_mg" else 1):
            inst.set_field("uv", np.zeros(2 * n_nodes))
            reps.append(inst.solve(cg_tol=1e-10 if a.case == "cg_mg" else 1e-6, outer_tol=1e300, max_outer=1,
                                   levels=1, precond=2, max_cg=100000))
        out.update(nodes=n_nodes, cg_iters=[r["cg_iters"] for r in reps], rel_res=reps[-1]["cg_rel_res"],
                   seconds=[r["seconds"] for r in reps], launches=reps[-1]["kernel_launches"])
        inst.close()
    elif a.case == "cg_fused_large":
        inst = _instance(ctx, 256, 1024)
        n_nodes = inst.sizes()[0]
        inst.set_field("uv", np.zeros(2 * n_nodes))
        rep = inst.solve(allow_not_converged=True, cg_tol=1e-12, outer_tol=1e300, max_outer=1, levels=1,
                         precond=1, max_cg=a.repeat)
        out.update(nodes=n_nodes, cg_iters=rep["cg_iters"], seconds=rep["seconds"],
                   launches=rep["kernel_launches"])
        inst.close()
    elif a.case in ("assemble", "update", "cg_large"):
        inst = _instance(ctx, 256, 1024)
        n_nodes, n_elem, nnz, _ = inst.sizes()
        out.update(nodes=n_nodes, elements=n_elem, nnz=nnz)
        if a.case == "assemble":
            ms, by = ctypes.c_double(), ctypes.c_double()
            ctx.check(C.lib().cp_bench_assemble(inst._h, CP_PREC_FP64, a.repeat, ctypes.byref(ms), ctypes.byref(by)))
            out.update(ms_per_launch=ms.value, bytes_per_launch=by.value)
        elif a.case == "update":
            inst.assemble(CP_PREC_FP64)
            it, _ = inst.cg_solve(1e-6)
            out["cg_iters"] = it
            out["rel_err"] = [inst.secant_update() for _ in range(a.repeat)]
        else:
            mp, mu, bp, bu = (ctypes.c_double() for _ in range(4))
            inst.set_field("uv", np.zeros(2 * n_nodes))
            prec = C.CP_PREC_MIXED if a.fp32 else CP_PREC_FP64
            ctx.check(C.lib().cp_bench_cg(inst._h, prec, 0, a.repeat, ctypes.byref(mp), ctypes.byref(mu),
                                          ctypes.byref(bp), ctypes.byref(bu)))
            out.update(ms_spmv=mp.value, ms_update=mu.value, bytes_spmv=bp.value, bytes_update=bu.value)
        inst.close()
    else:
        inst = _instance(ctx, 16, 64)
        reps = []
        for _ in range(a.repeat):
            inst.set_field("uv", np.zeros(2 * inst.sizes()[0]))
            reps.append(inst.solve(cg_tol=1e-10, outer_tol=1e300, max_outer=1, levels=1, precond=1,
                                   max_cg=100000))
        out.update(nodes=inst.sizes()[0], cg_iters=[r["cg_iters"] for r in reps],
                   rel_res=reps[-1]["cg_rel_res"], seconds=[r["seconds"] for r in reps],
                   us_per_iter=min(r["seconds"] / max(1, r["cg_iters"]) for r in reps) * 1e6)
        inst.close()
    ctx.close()
    print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
