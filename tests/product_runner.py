"""Runs a job in the harness syntax (see oracle/ref_harness.cu) through the
PRODUCT: the host-side drop-in classes build the mesh and the loads, and the
CUDA library solves, all through the C ABI. Used by the GPU parity tests so
that product and oracle see the identical job description."""
import numpy as np

import cudaplasticity_b200 as cp


def parse(lines):
    job = dict(mode="phases", E=None, nu=0.3, h=1.0, diagram=None, plane=cp.CP_PLANE_STRESS, cg_eps=1e-7,
               outer_eps=1e-5, max_outer=50, levels=1, loads=[])
    for ln in lines:
        w = ln.split()
        if not w or w[0].startswith("#"):
            continue
        k = w[0]
        if k == "mode":
            job["mode"] = w[1]
        elif k == "mesh":
            pass
        elif k == "material":
            job["E"], job["nu"], job["h"] = float(w[1]), float(w[2]), float(w[3])
        elif k == "diagram":
            job["diagram"] = w[1:]
        elif k == "plane":
            job["plane"] = cp.CP_PLANE_STRAIN if w[1] == "strain" else cp.CP_PLANE_STRESS
        elif k in ("cg_eps", "outer_eps"):
            job[k] = float(w[1])
        elif k in ("max_outer", "levels"):
            job[k] = int(w[1])
        elif k in ("dump_k", "dump_csr"):
            pass
        else:
            job["loads"].append(w)
    return job


def material_of(job):
    d = job["diagram"]
    E = job["E"] if job["E"] is not None else float(d[1])
    kw = dict(E=E, nu=job["nu"], h=job["h"], plane=job["plane"])
    if d is None:
        return cp.material(**kw)
    v = [float(x) for x in d[1:]] if d[0] != "piecewise" else None
    if d[0] == "linear":
        return cp.material(diagram="linear", sigma_t=v[1], k_t=v[2], **kw)
    if d[0] == "power":
        return cp.material(diagram="power", sigma_t=v[1], a=v[2], m=v[3], **kw)
    if d[0] == "hollomon":
        return cp.material(diagram="hollomon", sigma_y=v[1], eps0=v[2], n=v[3], **kw)
    if d[0] == "piecewise":
        n = int(d[2])
        vals = [float(x) for x in d[3:3 + 2 * n]]
        return cp.material(diagram="piecewise", points=list(zip(vals[0::2], vals[1::2])), **kw)
    raise ValueError(d)


def loads_of(job):
    L = cp.Loads()
    for w in job["loads"]:
        k, a = w[0], w[1:]
        f = [float(x) for x in a]
        if k == "force":
            L.set_force(int(a[0]), f[1], f[2], bool(int(a[3])))
        elif k == "fixborderhor":
            L.fix_border_hor(int(a[0]))
        elif k == "fixbordervert":
            L.fix_border_vert(int(a[0]))
        elif k == "fixvertaxis":
            L.fix_vert_axis(f[0])
        elif k == "fixhoraxis":
            L.fix_hor_axis(f[0])
        elif k == "fixpoint":
            L.fix_point(f[0], f[1])
        elif k == "displ":
            L.set_displacement(int(a[0]), f[1], f[2], bool(int(a[3])), bool(int(a[4])))
        elif k == "forcepoint":
            L.set_force_point(*f)
        elif k == "displpoint":
            L.set_displ_point(*f)
        elif k == "gravity":
            L.set_gravity(*f)
        elif k == "fixdof":
            L.fix_dof(int(a[0]))
        else:
            raise ValueError(k)
    return L


def build_inputs(lines, mesh_arrays):
    """rp, mask, uv from the product's host-side load builder."""
    job = parse(lines)
    mesh = cp.Mesh.from_arrays(mesh_arrays["node_xy"], mesh_arrays.get("elem3"), mesh_arrays.get("elem4"),
                               mesh_arrays["borders"], mesh_arrays.get("elem8"))
    return job, loads_of(job).build(mesh, h=job["h"], rho=1.0)


def run(ctx, lines, mesh_arrays, want_k=False, **solve_kw):
    """Returns the product's outputs under the oracle's record names."""
    job, (rp, mask, uv) = build_inputs(lines, mesh_arrays)
    inst = cp.Instance(ctx, mesh_arrays, material_of(job))
    inst.set_loads(rp, mask, uv)
    out = {"rp": rp, "mask": mask}
    if want_k:
        inst.assemble(cp.CP_PREC_FP64)
        out.update(inst.csr())
        out["slots"] = inst.slot_map()
    elastic = job["mode"] == "elastic"
    kw = dict(cg_tol=job["cg_eps"], outer_tol=1e300 if elastic else job["outer_eps"],
              max_outer=1 if elastic else job["max_outer"], levels=job["levels"])
    kw.update(solve_kw)
    rep = inst.solve(**kw)
    out.update(inst.state())
    out["report"] = rep
    inst.close()
    return out
