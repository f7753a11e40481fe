"""Pins of the oracle (the C restatement in oracle/) against the reference:
its golden fixtures (made by running the reference, tests/golden/make_golden.py)
and the result files shipped with the reference. CPU only."""
import json
import os

import numpy as np
import pytest

import meshgen
import oracle
import scenarios

from parity import FIELDS, field_error, rel_l2, yielded
REF_SCEN = [n for n, s in scenarios.SCENARIOS.items() if s.get("reference")]


def run_scenario(name, workdir, extra=()):
    path = os.path.join(workdir, f"{name}.bin")
    m, lines = scenarios.scenario_lines(name, path, extra=extra)
    oracle.write_mesh(path, m["node_xy"], elem3=m["elem3"], elem4=m["elem4"], borders=m["borders"],
                      elem8=m.get("elem8", ()))
    return m, oracle.run_oracle(lines)


@pytest.mark.parametrize("name", REF_SCEN)
def test_oracle_matches_reference_fixture(name, golden_dir, workdir):
    g = np.load(os.path.join(golden_dir, f"{name}.npz"))
    m, r = run_scenario(name, workdir, extra=["dump_k 1", "dump_csr 1"])
    assert scenarios.mesh_digest(m) == str(g["mesh_digest"])
    # integer work: bit-exact
    for k in ["rows", "cols", "adj_pos", "adj", "mask"]:
        assert np.array_equal(r[k], g[k]), k
    # the right-hand side and the first assembly are computed in the same
    # operation order as the reference's single-threaded run: bit-exact too.
    # 8-node elements: the oracle's Gauss constants carry full precision where
    # the reference writes 15 decimals, so their values agree to ~1e-15.
    assert np.array_equal(r["rp"], g["rp"])
    if "elem8" in m:
        assert np.max(np.abs(r["k_data"] - g["k_data"])) <= 1e-14 * np.max(np.abs(g["k_data"]))
    else:
        assert np.array_equal(r["k_data"], g["k_data"])
    # converged FP64 state under tight tolerances: 1e-10 relative L2
    for k in FIELDS:
        assert field_error(k, r, g) <= 1e-10, (k, field_error(k, r, g))
    # yielded set: elements on the plastic branch of the diagram (psi > 1)
    assert np.array_equal(yielded(r), yielded(g))


def test_meshgen_matches_reference_generators(golden_dir):
    ref = json.load(open(os.path.join(golden_dir, "ref_meshes.json")))
    makers = {
        "hole -3 3 -2 2 0.5 48 32 1": lambda: meshgen.hole_plate(-3, 3, -2, 2, 0.5, 48, 32),
        "hole -3 3 -2 2 0.5 12 8 1": lambda: meshgen.hole_plate(-3, 3, -2, 2, 0.5, 12, 8),
        "hole -100 100 -100 100 20 16 16 1": lambda: meshgen.hole_plate(-100, 100, -100, 100, 20, 16, 16),
        "ring 50 120 32 8 1": lambda: meshgen.ring(50, 120, 32, 8),
        "ring 0.1 0.2 40 5 1": lambda: meshgen.ring(0.1, 0.2, 40, 5),
        "rect -1 1 -1 1 4 4 1": lambda: meshgen.rect(-1, 1, -1, 1, 4, 4),
        "rect -3 3 -2 2 6 4 1": lambda: meshgen.rect(-3, 3, -2, 2, 6, 4),
    }
    for spec, mk in makers.items():
        assert scenarios.mesh_digest(mk()) == ref[spec]["digest"], spec


def test_oracle_vs_shipped_plasticity_vtk(golden_dir, workdir):
    """data/holePlatePlastPow.vtk (plasticityTest, src/Main.cpp:252-296) was
    written by the reference at its own tolerances (CG 1e-7, outer 1e-5); the
    oracle run the same way reproduces it to the same level the reference's
    CPU path does (about 1e-8), with the identical yielded set."""
    g = np.load(os.path.join(golden_dir, "ref_holePlatePlastPow.npz"))
    m = meshgen.hole_plate(-3, 3, -2, 2, 0.5, 48, 32)
    path = os.path.join(workdir, "m.bin")
    oracle.write_mesh(path, m["node_xy"], elem4=m["elem4"], borders=m["borders"])
    r = oracle.run_oracle(["mode solve", f"mesh file {path}", f"diagram power {scenarios.E304} 170 1930 0.015",
                           f"material {scenarios.E304} {scenarios.NU304} 1", "force 1 170 0 0", "force 3 -170 0 0",
                           "fixvertaxis 0", "fixhoraxis 0"])
    pairs = {"Eps_xx": "exx", "Eps_yy": "eyy", "Gamma_xy": "gamma", "Eps_intensity": "eps_i", "Eps_p_xx": "exx_p",
             "Eps_p_yy": "eyy_p", "Gamma_p_xy": "gamma_p", "Eps_p_intensity": "eps_p_i", "Psi": "psi", "E_c": "E_c",
             "nu_c": "nu_c", "Sigma_xx": "sxx", "Sigma_yy": "syy", "Tau_xy": "tau", "Sigma_intensity": "sig_i"}
    for vk, ok in pairs.items():
        assert rel_l2(r[ok], g[vk]) < 2e-7, (vk, rel_l2(r[ok], g[vk]))
    assert rel_l2(r["uv"], g["displacement"]) < 2e-8
    assert np.array_equal(r["psi"] > 1.0 + 1e-9, g["Psi"] > 1.0 + 1e-9)
    assert int((g["Psi"] > 1.0 + 1e-9).sum()) == 3528


def test_oracle_vs_shipped_patch_vtk(golden_dir, workdir):
    """data/solverTest.vtk (solverTest, src/Main.cpp:14-38)."""
    g = np.load(os.path.join(golden_dir, "ref_solverTest.npz"))
    _, r = run_scenario("rect_elastic", workdir)
    assert rel_l2(r["uv"], g["displacement"]) < 1e-10
    assert rel_l2(r["sxx"], g["Sigma_xx"]) < 1e-10
    assert rel_l2(r["exx"], g["Eps_xx"]) < 1e-10
    assert rel_l2(r["sig_i"], g["Sigma_intensity"]) < 1e-10


@pytest.mark.parametrize("table,diag,S", [
    ("aitken_plast1pow", f"diagram power {scenarios.E304 * 1e6} 170e6 {scenarios.E304 * 1e4} 0.015", 170e6),
    ("aitken_plast1", f"diagram linear {scenarios.E304 * 1e6} 170e6 {scenarios.E304 * 1e5}", 170e6),
    ("aitken_elast1", f"diagram power {scenarios.E304 * 1e6} 170e6 {scenarios.E304 * 1e4} 0.015", 1e6),
])
def test_oracle_energy_tables(table, diag, S, golden_dir, workdir):
    """data/aitken_*.txt (energyConvTest, src/Main.cpp:110-175): the strain
    energy of the 2880-element Q4 plate, printed with 6 significant digits."""
    tables = json.load(open(os.path.join(golden_dir, "ref_tables.json")))
    expected = [e for n, e in tables[table] if n == 2880][0]
    m = meshgen.hole_plate(-3, 3, -2, 2, 0.5, 36, 24)
    assert m["elem4"].shape[0] == 2880
    path = os.path.join(workdir, "m.bin")
    oracle.write_mesh(path, m["node_xy"], elem4=m["elem4"], borders=m["borders"])
    r = oracle.run_oracle(["mode solve", f"mesh file {path}", diag, f"material {scenarios.E304 * 1e6} 0.29 1",
                           f"force 1 {S} 0 0", f"force 3 {-S} 0 0", "fixvertaxis 0", "fixhoraxis 0"])
    got = float(r["energy"][0])
    assert float(f"{got:.6g}") == pytest.approx(expected, rel=1e-12), (got, expected)


@pytest.mark.parametrize("table,diag,S", [
    ("aitken_plast2pow", f"diagram power {scenarios.E304 * 1e6} 170e6 {scenarios.E304 * 1e4} 0.015", 170e6),
    ("aitken_plast2", f"diagram linear {scenarios.E304 * 1e6} 170e6 {scenarios.E304 * 1e5}", 170e6),
    ("aitken_elast2", f"diagram power {scenarios.E304 * 1e6} 170e6 {scenarios.E304 * 1e4} 0.015", 1e6),
])
def test_oracle_energy_tables_q8(table, diag, S, golden_dir, workdir):
    """The same energy tables for 8-node elements (energyConvTest with order 2,
    src/Main.cpp:110-175): the 2880-element Q8 plate. For Q8 elements the
    reference's deformEnergy takes the secant energy on both branches."""
    import cudaplasticity_b200 as cp

    tables = json.load(open(os.path.join(golden_dir, "ref_tables.json")))
    expected = [e for n, e in tables[table] if n == 2880][0]
    m = cp.Mesh.rect_with_hole(-3, 3, -2, 2, 0.5, 36, 24, order=2).arrays()
    assert m["elem8"].shape[0] == 2880 and m["elem4"].shape[0] == 0
    path = os.path.join(workdir, "m8.bin")
    oracle.write_mesh(path, m["node_xy"], borders=m["borders"], elem8=m["elem8"])
    r = oracle.run_oracle(["mode solve", f"mesh file {path}", diag, f"material {scenarios.E304 * 1e6} 0.29 1",
                           f"force 1 {S} 0 0", f"force 3 {-S} 0 0", "fixvertaxis 0", "fixhoraxis 0"])
    got = float(r["energy"][0])
    assert float(f"{got:.6g}") == pytest.approx(expected, rel=1e-12), (got, expected)


@pytest.mark.parametrize("name", ["hole_q8", "ring_q8", "rect_q8", "rect_points", "ring_mixed"])
def test_oracle_q8_loads(name, golden_dir, workdir):
    """The oracle's load builder on 8-node meshes (quadratic edges, 8-node
    body forces) and with the point and whole-border conditions, against the
    reference's initConditions on the same meshes."""
    import sys

    import cudaplasticity_b200 as cp

    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)) + "/golden")
    from make_golden import MISC_LOADS, Q8_LOADS

    g = dict(np.load(os.path.join(golden_dir, "q8_loads.npz")))
    spec, lines = {**Q8_LOADS, **MISC_LOADS}[name]
    w = spec.split()
    f = [float(x) for x in w[1:]]
    if w[0] == "hole":
        mesh = cp.Mesh.rect_with_hole(*f[:5], int(f[5]), int(f[6]), order=int(f[7]))
    elif w[0] == "ring":
        mesh = cp.Mesh.ring(f[0], f[1], int(f[2]), int(f[3]), order=int(f[4]))
    else:
        mesh = cp.Mesh.rect(*f[:4], int(f[4]), int(f[5]), order=int(f[6]))
    m = mesh.arrays()
    path = os.path.join(workdir, "l8.bin")
    oracle.write_mesh(path, m["node_xy"], elem4=m["elem4"], borders=m["borders"], elem8=m.get("elem8", ()))
    r = oracle.run_oracle(["mode elastic", f"mesh file {path}", "cg_eps 1e-3"] + lines)
    ref = g[f"{name}_rp"]
    assert np.max(np.abs(r["rp"] - ref)) <= 1e-14 * np.max(np.abs(ref))
    assert np.array_equal(r["mask"].astype(bool), g[f"{name}_mask"].astype(bool))


def test_oracle_diagram_reproduction(golden_dir, workdir):
    """data/diagramPow.txt (diagramTest, src/Main.cpp:929-994): a 2x2 patch
    pulled by imposed displacement reproduces the power-law diagram."""
    tables = json.load(open(os.path.join(golden_dir, "ref_tables.json")))
    expected = tables["diagramPow"]
    m = meshgen.rect(-1, 1, -1, 1, 2, 2)
    path = os.path.join(workdir, "m.bin")
    oracle.write_mesh(path, m["node_xy"], elem4=m["elem4"], borders=m["borders"])
    displ, rows = 0.0, []
    while displ <= 0.02:
        r = oracle.run_oracle(["mode solve", f"mesh file {path}",
                               f"diagram power {scenarios.E304 * 1e6} 170e6 {scenarios.E304 * 1e4} 0.015",
                               f"material {scenarios.E304 * 1e6} 0.29 1", "gravity 9.81 0 -1",
                               "displ 2 0 0 0 1", f"displ 0 {displ!r} 0 0 1"])
        rows.append((float(r["exx"][0]), float(r["sxx"][0]) * 1e-6))
        displ += 0.0005
    assert len(rows) == len(expected) == 40
    for (e, s), (ee, es) in zip(rows[1:], expected[1:]):
        assert float(f"{e:.6g}") == pytest.approx(ee, rel=1e-12)
        assert float(f"{s:.6g}") == pytest.approx(es, rel=1e-12)


def test_oracle_t3_patch(workdir):
    """CST extension: uniform tension of a triangulated rectangle gives the
    exact uniform stress (patch test) and E*eps = sigma in every element."""
    m = meshgen.split_t3(meshgen.rect(0.0, 4.0, 0.0, 2.0, 4, 2))
    path = os.path.join(workdir, "t3.bin")
    oracle.write_mesh(path, m["node_xy"], elem3=m["elem3"], borders=m["borders"])
    r = oracle.run_oracle(["mode elastic", f"mesh file {path}", "material 1000 0.25 1", "cg_eps 1e-14",
                           "force 0 3 0 0", "fixbordervert 2", "fixpoint 0 0"])
    assert np.allclose(r["sxx"], 3.0, rtol=1e-9, atol=1e-9)
    assert np.allclose(r["syy"], 0.0, atol=1e-8)
    assert np.allclose(r["tau"], 0.0, atol=1e-8)
    assert np.allclose(r["exx"], 3.0 / 1000, rtol=1e-9)
    assert np.allclose(r["eyy"], -0.25 * 3.0 / 1000, rtol=1e-9)


@pytest.mark.skipif(not os.path.exists(oracle.REF_BIN_CSR), reason="reference harness (cpref_csr) not built")
def test_reference_csr_direct_assembly_matches_band_assembly(golden_dir, workdir):
    """The CPU baseline of the 2.1M-DOF plate assembles the reference's own
    element matrices straight into CSR (mode phases_csr of the harness,
    built with the solver's source) because the reference's band matrix does
    not fit in host memory there. On a mesh where both fit, the converged
    state of the two assemblies agrees to round-off, with the same iteration
    counts, and matches the reference fixture; prefix_outer stops the run
    after that many outer iterations in all."""
    name = "ogrid16_bilin"
    path = os.path.join(workdir, f"{name}.bin")
    m, lines = scenarios.scenario_lines(name, path)
    oracle.write_mesh(path, m["node_xy"], elem4=m["elem4"], borders=m["borders"])
    csr = [ln.replace("mode phases", "mode phases_csr") for ln in lines]
    r = oracle.run_reference(csr, binary=oracle.REF_BIN_CSR)
    g = np.load(os.path.join(golden_dir, f"{name}.npz"))
    for k in FIELDS:
        assert field_error(k, r, g) <= 1e-12, (k, field_error(k, r, g))
    assert np.array_equal(r["outer_per_level"], g["outer_per_level"])
    assert r["cg_seconds"][0] > 0 and r["assembly_seconds"][0] > 0
    p = oracle.run_reference(csr + ["prefix_outer 8"], binary=oracle.REF_BIN_CSR)
    assert int(np.sum(p["outer_per_level"])) == 8
