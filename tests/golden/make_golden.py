"""Regenerates the golden fixtures in this directory from the reference.

Run from the repository root with CUPLAST_REFERENCE set to the reference
checkout (``CUPLAST_REFERENCE=<dir> python tests/golden/make_golden.py``); it builds the harness
(oracle/_ref/cpref) from them if needed. The fixtures it writes are:

* ``<scenario>.npz`` -- for every reference scenario in tests/scenarios.py:
  the reference's CSR structure, right-hand side, Dirichlet mask, the values
  of its first stiffness assembly (run with one thread, so the summation order
  is the element order) and its converged state under tight tolerances;
* ``config1_bilin.npz``, ``ogrid128x64_hollomon.npz`` -- configuration-size
  scenarios: the reference's converged state (tight tolerances) of the
  fields in scenarios.STATE_FIELDS;
* ``ref_meshes.json`` -- SHA-256 digests of meshes made by the reference's own
  generators (genRectWithHole, genRing, genRectangle);
* ``ref_holePlatePlastPow.npz`` and ``ref_solverTest.npz`` -- the cell fields
  and displacements of the VTK results shipped with the reference
  (data/holePlatePlastPow.vtk, data/solverTest.vtk);
* ``ref_tables.json`` -- the strain energies of data/aitken_*.txt and the
  stress-strain points of data/diagramPow.txt / diagramLin.txt;
* ``inp_<name>.inp`` and ``inp_<name>.npz`` -- small .inp mesh files written
  here (the reference ships none) and the arrays the reference's own
  Mesh::loadFromFile makes of them.
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle  # noqa: E402
import scenarios  # noqa: E402
from oracle import vtk  # noqa: E402

REF = os.environ.get("CUPLAST_REFERENCE", "")
OUT = os.path.dirname(os.path.abspath(__file__))
FIELDS = ["uv", "exx", "eyy", "gamma", "eps_i", "sxx", "syy", "tau", "sig_i", "table_s", "psi", "E_c", "nu_c",
          "exx_p", "eyy_p", "gamma_p", "eps_p_i"]


def scenario_fixtures(workdir, only=None):
    for name, sc in scenarios.SCENARIOS.items():
        if not sc.get("reference") or (only and name not in only):
            continue
        mesh_path = os.path.join(workdir, f"{name}.bin")
        m, lines = scenarios.scenario_lines(name, mesh_path, extra=["dump_k 1", "dump_csr 1"])
        oracle.write_mesh(mesh_path, m["node_xy"], elem3=m["elem3"], elem4=m["elem4"], borders=m["borders"],
                          elem8=m.get("elem8", ()))
        r = oracle.run_reference(lines, threads=1)
        arrays = {k: r[k] for k in ["rows", "cols", "adj_pos", "adj", "rp", "mask", "k_data"] + FIELDS}
        arrays.update(outer_per_level=r["outer_per_level"], cg_per_level=r["cg_per_level"],
                      err_per_level=r["err_per_level"], energy=r["energy"],
                      mesh_digest=np.array(scenarios.mesh_digest(m)))
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **arrays)
        print(name, "outer", r["outer_per_level"], "cg", r["cg_per_level"])


def state_fixtures(workdir, only=None):
    """Configuration-size scenarios: the reference's converged state under
    tight tolerances (all host threads), STATE_FIELDS only, float64."""
    for name, sc in scenarios.SCENARIOS.items():
        if not sc.get("state_fixture") or (only and name not in only):
            continue
        mesh_path = os.path.join(workdir, f"{name}.bin")
        m, lines = scenarios.scenario_lines(name, mesh_path)
        oracle.write_mesh(mesh_path, m["node_xy"], elem3=m["elem3"], elem4=m["elem4"], borders=m["borders"])
        r = oracle.run_reference(lines)
        arrays = {k: r[k] for k in scenarios.STATE_FIELDS}
        arrays.update(outer_per_level=r["outer_per_level"], cg_per_level=r["cg_per_level"],
                      err_per_level=r["err_per_level"], mesh_digest=np.array(scenarios.mesh_digest(m)))
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **arrays)
        print(name, "outer", r["outer_per_level"], "cg", r["cg_per_level"])


def mesh_fixtures():
    specs = ["hole -3 3 -2 2 0.5 48 32 1", "hole -3 3 -2 2 0.5 12 8 1", "hole -100 100 -100 100 20 16 16 1",
             "ring 50 120 32 8 1", "ring 0.1 0.2 40 5 1", "rect -1 1 -1 1 4 4 1", "rect -3 3 -2 2 6 4 1",
             # 8-node (order 2) meshes: Mesh::remapOrder
             "hole -3 3 -2 2 0.5 12 8 2", "ring 50 120 16 4 2", "rect -3 3 -2 2 6 4 2"]
    out = {}
    for s in specs:
        r = oracle.run_reference(["mode mesh", "mesh " + s])
        off, borders = 0, []
        for L in r["border_len"]:
            borders.append(r["border_nodes"][off:off + L])
            off += L
        m = dict(node_xy=r["node_xy"].reshape(-1, 2), elem3=r["elem3"], elem4=r["elem4"], borders=borders,
                 elem8=r["elem8"], sec_ord=r["sec_ord"])
        out[s] = dict(digest=scenarios.mesh_digest(m), nodes=int(len(r["node_xy"]) // 2),
                      count4=int(len(r["elem4"]) // 4), max_index_diff=int(r["max_index_diff"][0]),
                      **({"count8": int(len(r["elem8"]) // 8)} if len(r["elem8"]) else {}))
    with open(os.path.join(OUT, "ref_meshes.json"), "w") as f:
        json.dump(out, f, indent=1)


def shipped_fixtures():
    v = vtk.read_solution_vtk(os.path.join(REF, "data", "holePlatePlastPow.vtk"))
    np.savez_compressed(os.path.join(OUT, "ref_holePlatePlastPow.npz"),
                        displacement=v["point_fields"]["Displacement"][:, :2].ravel(), **v["cell_fields"])
    v = vtk.read_solution_vtk(os.path.join(REF, "data", "solverTest.vtk"))
    np.savez_compressed(os.path.join(OUT, "ref_solverTest.npz"),
                        displacement=v["point_fields"]["Displacement"][:, :2].ravel(), **v["cell_fields"])
    tables = {}
    for name in ["aitken_plast1pow", "aitken_plast1", "aitken_elast1", "aitken_plast2pow", "aitken_plast2",
                 "aitken_elast2"]:
        rows = []
        with open(os.path.join(REF, "data", name + ".txt")) as f:
            next(f)
            for line in f:
                w = line.split()
                rows.append([int(w[0]), float(w[1])])
        tables[name] = rows
    for name in ["diagramPow", "diagramLin"]:
        with open(os.path.join(REF, "data", name + ".txt")) as f:
            tables[name] = [[float(w) for w in line.split()] for line in f if line.strip()]
    with open(os.path.join(OUT, "ref_tables.json"), "w") as f:
        json.dump(tables, f, indent=1)


# Load building on 8-node meshes (quadratic edges, 8-node body forces):
# name -> (reference mesh spec, job lines)
Q8_LOADS = {
    "hole_q8": ("hole -3 3 -2 2 0.5 12 8 2",
                ["material 193000 0.29 1", "force 1 170 0 0", "force 3 -170 0 0", "fixvertaxis 0", "fixhoraxis 0"]),
    "ring_q8": ("ring 50 120 16 4 2",
                ["material 210000 0.3 1", "force 0 200 0 1", "fixborderhor 1", "gravity 9.81 0 -1"]),
    "rect_q8": ("rect -3 3 -2 2 6 4 2",
                ["material 210000 0.3 2", "force 0 0 -50 0", "displ 2 0 0 0 0", "gravity 2.5 1 0"]),
}


# The remaining load and boundary-condition setters on 4-node meshes: point
# forces, prescribed point displacements (fixPoint / setDisplPoint), whole
# borders prescribed (setDisplacement without the mid-point options,
# fixBorder), one-axis border fixes, plane strain, a thickness other than 1.
MISC_LOADS = {
    "rect_points": ("rect -2 2 -1 1 8 4 1",
                    ["material 1000 0.25 1.5", "plane strain", "forcepoint 2 1 3 -4", "forcepoint 0 -1 0 -7.5",
                     "displpoint -2 -1 0.01 -0.02", "fixpoint -2 1", "displ 1 0.05 0 0 0", "fixbordervert 3",
                     "force 2 0 -10 0"]),
    "ring_mixed": ("ring 50 120 24 6 1",
                   ["material 210000 0.3 2", "force 0 150 20 1", "displ 1 0 0 0 0", "forcepoint 120 0 0 500",
                    "gravity 9.81 1 1"]),
}


# Mesh tooling: (reference mesh spec, operations applied after it)
MESH_TOOLS = {
    "hole_renum11": ("hole -3 3 -2 2 0.5 12 8 1", [("renum", 1.0, 1.0)]),
    "ring_q8_renum": ("ring 50 120 16 4 2", [("renum", 0.3, -1.0)]),
    "ogrid_smooth": ("hole -100 100 -100 100 20 8 8 1", [("smooth_ring", 32)]),
    "rect_renum_ties": ("rect -3 3 -2 2 6 4 1", [("renum", 1.0, 0.0)]),
}


def mesh_tool_fixtures():
    out = {}
    for name, (spec, ops) in MESH_TOOLS.items():
        r = oracle.run_reference(["mode mesh", "mesh " + spec] + [" ".join(str(x) for x in op) for op in ops])
        off, borders = 0, []
        for L in r["border_len"]:
            borders.append(r["border_nodes"][off:off + L])
            off += L
        m = dict(node_xy=r["node_xy"].reshape(-1, 2), elem3=r["elem3"], elem4=r["elem4"], borders=borders,
                 elem8=r["elem8"], sec_ord=r["sec_ord"])
        out[f"{name}_digest"] = np.array(scenarios.mesh_digest(m))
        for k in ("aspect", "skew_sin", "avr_elem_size"):
            out[f"{name}_{k}"] = r[k]
    np.savez_compressed(os.path.join(OUT, "ref_mesh_tools.npz"), **out)
    print("mesh tools", list(MESH_TOOLS))


def q8_load_fixtures():
    out = {}
    for name, (spec, lines) in list(Q8_LOADS.items()) + list(MISC_LOADS.items()):
        r = oracle.run_reference(["mode loads", "mesh " + spec] + lines)
        for k in ("rp", "mask", "uv"):
            out[f"{name}_{k}"] = r[k]
    np.savez_compressed(os.path.join(OUT, "q8_loads.npz"), **out)
    print("q8 loads", list(Q8_LOADS))


def write_inp_files():
    """Two .inp inputs: ``mixed`` (a 12 x 8 O-grid plate with every other quad
    split into triangles, nodes listed out of order, four *MPC border blocks
    with one reference node each, comment lines between sections) and
    ``quirks`` (a section header right after a block's last data line, which
    the reference's reader consumes with the block, a blank-line terminator,
    comma-free lines, a file that ends inside an *MPC block)."""
    sys.path.insert(0, ROOT)
    import cudaplasticity_b200 as cp

    m = cp.Mesh.rect_with_hole(-3.0, 3.0, -2.0, 2.0, 0.5, 12, 8).arrays()
    xy, e4, borders = m["node_xy"], m["elem4"], m["borders"]
    n = len(xy)
    tri, quad = [], []
    for k, q in enumerate(e4):
        if k % 2 == 0:
            tri += [(q[0], q[1], q[2]), (q[0], q[2], q[3])]
        else:
            quad.append(tuple(q))
    rng = np.random.default_rng(5)
    order = rng.permutation(n)
    L = ["*HEADING", "mixed S3/S4 mesh for the loader pins", "*NODE"]
    L += [f"{i + 1:6d}, {float(xy[i, 0])!r}, {float(xy[i, 1])!r}" for i in order]
    L += [f"{n + b + 1:6d}, 0.0, 0.0" for b in range(len(borders))]  # one reference node per *MPC block
    L += ["**", "*ELEMENT, TYPE=S3, ELSET=TRI"]
    L += [f"{k + 1}, {a + 1}, {b + 1}, {c + 1}" for k, (a, b, c) in enumerate(tri)]
    L += ["**", "*ELEMENT, TYPE=S4R, ELSET=QUAD"]
    L += [f"{len(tri) + k + 1}, " + ", ".join(str(v + 1) for v in q) for k, q in enumerate(quad)]
    L += ["**"]
    for b, nodes in enumerate(borders):
        L += ["*MPC"] + [f"BEAM, {v + 1}, {n + b + 1}" for v in nodes]
    L += ["**", "*END"]
    with open(os.path.join(OUT, "inp_mixed.inp"), "w") as f:
        f.write("\n".join(L) + "\n")

    r = cp.Mesh.rect(0.0, 2.0, 0.0, 1.0, 4, 2).arrays()
    xy, e4, borders = r["node_xy"], r["elem4"], r["borders"]
    n = len(xy)
    L = ["*NODE"] + [f"{i + 1} {float(xy[i, 0])!r} {float(xy[i, 1])!r}" for i in range(n)]
    L += [f"{n + b + 1} 9.0 9.0" for b in range(2)]
    L += ["*ELEMENT, TYPE=S3"]  # consumed as the terminator of the *NODE block: its data lines are skipped
    L += ["1, 1, 2, 3"]
    L += ["", "*ELEMENT, TYPE=S4"] + [f"{k + 1} " + " ".join(str(v + 1) for v in q) for k, q in enumerate(e4)]
    L += ["", "*MPC"] + [f"BEAM, {v + 1}, {n + 1}" for v in borders[0]]
    L += ["*MPC"] + [f"BEAM, {v + 1}, {n + 2}" for v in borders[2]]
    with open(os.path.join(OUT, "inp_quirks.inp"), "w") as f:
        f.write("\n".join(L) + "\n")


def inp_fixtures():
    write_inp_files()
    for name in ["mixed", "quirks"]:
        r = oracle.run_reference(["mode mesh", "mesh inp " + os.path.join(OUT, f"inp_{name}.inp")],
                                 binary=oracle.REF_BIN_INP)
        np.savez_compressed(os.path.join(OUT, f"inp_{name}.npz"),
                            **{k: r[k] for k in ["node_xy", "elem3", "elem4", "elem8", "border_len", "border_nodes"]})
        print("inp", name, "nodes", len(r["node_xy"]) // 2, "tri", len(r["elem3"]) // 3, "quad", len(r["elem4"]) // 4,
              "borders", list(r["border_len"]))


if __name__ == "__main__":
    import tempfile

    if not REF or not os.path.isdir(os.path.join(REF, "src")):
        sys.exit("set CUPLAST_REFERENCE to the reference checkout (its src/ and data/ are read)")

    if "--meshes" in sys.argv:  # only the generator and load-building pins
        if not oracle.have_reference():
            oracle.build(with_reference=True, ref_dir=REF)
        mesh_fixtures()
        q8_load_fixtures()
        mesh_tool_fixtures()
        sys.exit(0)
    if "--scenarios" in sys.argv:  # only the named scenario fixtures
        if not oracle.have_reference():
            oracle.build(with_reference=True, ref_dir=REF)
        with tempfile.TemporaryDirectory() as d:
            scenario_fixtures(d, only=sys.argv[sys.argv.index("--scenarios") + 1:])
        sys.exit(0)
    if "--states" in sys.argv:  # only the configuration-size state fixtures
        if not oracle.have_reference():
            oracle.build(with_reference=True, ref_dir=REF)
        with tempfile.TemporaryDirectory() as d:
            state_fixtures(d, only=sys.argv[sys.argv.index("--states") + 1:])
        sys.exit(0)
    if "--inp" in sys.argv:  # only the .inp loader pins
        if not oracle.have_reference():
            oracle.build(with_reference=True, ref_dir=REF)
        inp_fixtures()
        sys.exit(0)

    if not oracle.have_reference():
        oracle.build(with_reference=True, ref_dir=REF)
    with tempfile.TemporaryDirectory() as d:
        scenario_fixtures(d)
        state_fixtures(d)
    mesh_fixtures()
    q8_load_fixtures()
    mesh_tool_fixtures()
    shipped_fixtures()
    inp_fixtures()
