"""The drop-in C++ classes (include/cuplast/*.hpp), used the way a user of the
reference uses them: tests/cxx/scenario_drivers.cpp restates scenarios of the
reference's src/Main.cpp against them, built here with g++ and linked to the
in-tree libcuplast.so.

CPU: the drivers compile and link against the headers and the library, and
without a device they fail with the library's message instead of crashing.
GPU: the files and numbers they write agree with what the reference shipped
for the same scenarios (data/solverTest.vtk, data/holePlatePlastPow.vtk,
data/aitken_*.txt)."""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import vtk
from parity import rel_l2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cxx", "scenario_drivers.cpp")
LIBDIR = os.path.join(ROOT, "cudaplasticity_b200")


@pytest.fixture(scope="module")
def drivers(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    if not os.path.exists(os.path.join(LIBDIR, "libcuplast.so")):
        pytest.skip("libcuplast.so not built")
    exe = str(tmp_path_factory.mktemp("cxx") / "scenario_drivers")
    subprocess.run([gxx, "-std=c++17", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"), SRC, "-L" + LIBDIR,
                    "-lcuplast", "-Wl,-rpath," + LIBDIR, "-o", exe], check=True)
    return exe


def test_drivers_build_and_fail_cleanly_without_a_device(drivers):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([drivers, "noDevice"], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0, (r.stdout, r.stderr)
    assert "error: cuplast: no CUDA device" in r.stdout
    r = subprocess.run([drivers], capture_output=True, text=True, timeout=60)
    assert r.returncode == 64 and "usage" in r.stderr


def test_mesh_tooling_through_the_drop_in_classes(drivers, tmp_path):
    """Mesh::renumByDirection, printAnalysis, the copy constructor and the
    mesh VTK writer (src/Mesh.cu:939-990, 1032-1080) from C++, host only: the
    file lists the mesh with the analysis fields, consistent with the same
    mesh through the C ABI."""
    import cudaplasticity_b200 as cp

    out = str(tmp_path / "mesh.vtk")
    r = subprocess.run([drivers, "meshVtk", out], capture_output=True, text=True, check=True, timeout=120)
    assert "Mesh analysis:" in r.stdout and "Aspect ratio" in r.stdout
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("avr ")][0].split()
    m = cp.Mesh.rect_with_hole(-3, 3, -2, 2, 0.5, 12, 8).renum_by_direction(1.0, 1.0)
    q = m.quality()
    assert float(line[1]) == q["avr_elem_size"] and int(line[3]) == m.max_index_diff()
    tok = open(out).read().split()
    n, c4 = m.counts()[0], m.counts()[2]
    assert tok[tok.index("POINTS") + 1] == str(n) and tok[tok.index("POLYGONS") + 1] == str(c4)
    assert tok[tok.index("FieldData") + 1] == "3"
    i = tok.index("Element_aspect_ratio")
    aspect = np.array([float(x) for x in tok[i + 4:i + 4 + c4]])
    assert np.allclose(aspect, q["aspect"], rtol=1e-5)
    i = tok.index("Element_skew_angle")
    skew = np.array([float(x) for x in tok[i + 4:i + 4 + c4]])
    assert np.allclose(skew, np.arccos(q["skew_sin"]), rtol=1e-5, atol=1e-6)


@pytest.mark.gpu
def test_solver_test_vtk_matches_reference(drivers, golden_dir, tmp_path):
    """solverTest (src/Main.cpp:14-38) through the drop-in classes: the VTK
    written by saveAsVtk against data/solverTest.vtk."""
    out = str(tmp_path / "solverTest.vtk")
    subprocess.run([drivers, "solverTest", out], check=True, timeout=300)
    v = vtk.read_solution_vtk(out)
    g = np.load(os.path.join(golden_dir, "ref_solverTest.npz"))
    assert rel_l2(v["point_fields"]["Displacement"][:, :2].ravel(), g["displacement"]) < 1e-10
    for k in ["Sigma_xx", "Eps_xx", "Sigma_intensity"]:
        assert rel_l2(v["cell_fields"][k], g[k]) < 1e-10, k


@pytest.mark.gpu
def test_plasticity_test_vtk_matches_reference(drivers, golden_dir, tmp_path):
    """plasticityTest (src/Main.cpp:252-296) through the drop-in classes, at
    the reference's own tolerances: the VTK written by saveAsVtk against
    data/holePlatePlastPow.vtk, to the level the reference's CPU path
    reproduces it (the oracle test of the same file has the same bars)."""
    out = str(tmp_path / "holePlatePlastPow.vtk")
    subprocess.run([drivers, "plasticityTest", out], check=True, timeout=600)
    v = vtk.read_solution_vtk(out)
    g = np.load(os.path.join(golden_dir, "ref_holePlatePlastPow.npz"))
    assert set(g.files) - {"displacement"} <= set(v["cell_fields"]) | {"ElementID"}
    for k in [f for f in g.files if f != "displacement"]:
        assert rel_l2(v["cell_fields"][k], g[k]) < 2e-7, (k, rel_l2(v["cell_fields"][k], g[k]))
    assert rel_l2(v["point_fields"]["Displacement"][:, :2].ravel(), g["displacement"]) < 2e-8
    assert np.array_equal(v["cell_fields"]["Psi"] > 1.0 + 1e-9, g["Psi"] > 1.0 + 1e-9)


def _six_digits(got, expected):
    """The reference prints energies with 6 significant digits; a value within
    a hair of a rounding boundary may print either way."""
    digit = 10.0 ** (np.floor(np.log10(abs(expected))) - 5)
    return abs(got - expected) <= 0.5 * digit * (1 + 1e-6) + 1e-7 * abs(expected)


@pytest.mark.gpu
@pytest.mark.parametrize("order,kind,table", [(2, "power", "aitken_plast2pow"), (2, "linear", "aitken_plast2"),
                                              (2, "elastic", "aitken_elast2"), (1, "power", "aitken_plast1pow")])
def test_energy_conv_test_energies(drivers, golden_dir, order, kind, table):
    """energyConvTest (src/Main.cpp:110-175) on its 2880-element plate through
    the drop-in classes: deformEnergy against data/aitken_*.txt, for 8-node
    (order 2) and 4-node elements."""
    r = subprocess.run([drivers, "energyConvTest", str(order), kind], capture_output=True, text=True, check=True,
                       timeout=600)
    w = r.stdout.split()
    assert w[0] == "elements" and int(w[1]) == 2880
    got = float(w[3])
    tables = json.load(open(os.path.join(golden_dir, "ref_tables.json")))
    expected = [e for n, e in tables[table] if n == 2880][0]
    assert _six_digits(got, expected), (got, expected)


def _polar(c, x, y, xy):
    """_rr, _phiphi, _rphi of src/PlasticitySolver.cuh:169-200 at centres c."""
    r = np.sqrt(c[:, 0] ** 2 + c[:, 1] ** 2)
    cs, sn = c[:, 0] / r, c[:, 1] / r
    return (cs * cs * x + sn * sn * y + 2.0 * cs * sn * xy, sn * sn * x + cs * cs * y - 2.0 * cs * sn * xy,
            cs * sn * (-x + y) + xy * (cs * cs - sn * sn))


@pytest.mark.gpu
@pytest.mark.parametrize("segments", [4, 8])
def test_kirsch_error_norms_and_polar_vtk(drivers, segments, tmp_path):
    """kirschConvTest (src/Main.cpp:178-227) through the drop-in classes:
    polarSigmaError and sigmaError (src/PlasticitySolver.cuh:464-540) and the
    polar-coordinate VTK, against the same formulas applied here (numpy) to
    the oracle's solution of the same elastic problem."""
    import meshgen
    import oracle

    out = str(tmp_path / "kirsch.vtk")
    r = subprocess.run([drivers, "kirschTest", str(segments), out], capture_output=True, text=True, check=True,
                       timeout=300)
    w = r.stdout.split()
    assert w[0] == "polar" and w[2] == "cartesian_zero"
    polar_err, cart_err = float(w[1]), float(w[3])
    m = meshgen.hole_plate(-3, 3, -2, 2, 0.5, segments, segments)
    path = str(tmp_path / "m.bin")
    oracle.write_mesh(path, m["node_xy"], elem4=m["elem4"], borders=m["borders"])
    S, a, E, nu = 1e6, 0.5, 193e9, 0.29
    o = oracle.run_oracle(["mode elastic", f"mesh file {path}", f"material {E} {nu} 1", "cg_eps 1e-13",
                           f"force 1 {S} 0 0", f"force 3 {-S} 0 0", "fixvertaxis 0", "fixhoraxis 0"])
    xy, e4 = np.asarray(m["node_xy"]), np.asarray(m["elem4"])
    p = xy[e4]
    c = (((p[:, 0] + p[:, 1]) + p[:, 2]) + p[:, 3]) / 4
    x, y = p[:, :, 0], p[:, :, 1]
    area = np.abs((x * np.roll(y, -1, axis=1)).sum(1) - (y * np.roll(x, -1, axis=1)).sum(1)) * 0.5
    sxx, syy, tau = o["sxx"], o["syy"], o["tau"]
    # polarSigmaError against Kirsch's solution, centres within r <= 2
    rr, pp, rp = _polar(c, sxx, syy, tau)
    rad = np.sqrt(c[:, 0] ** 2 + c[:, 1] ** 2)
    phi = np.arctan(c[:, 1] / c[:, 0]) + np.where(c[:, 0] < 0, np.pi, 0.0)
    s_r = 0.5 * S * (1 - a * a / rad ** 2) + 0.5 * S * (1 + 3 * a ** 4 / rad ** 4 - 4 * a * a / rad ** 2) * np.cos(2 * phi)
    s_p = 0.5 * S * (1 + a * a / rad ** 2) - 0.5 * S * (1 + 3 * a ** 4 / rad ** 4) * np.cos(2 * phi)
    s_rp = -0.5 * S * (1 - 3 * a ** 4 / rad ** 4 + 2 * a * a / rad ** 2) * np.sin(2 * phi)
    k = rad <= 2.0
    vol = area[k].sum()
    expect_polar = max(np.abs(s_r - rr)[k].max() * vol / (np.abs(rr) * area)[k].sum(),
                       np.abs(s_p - pp)[k].max() * vol / (np.abs(pp) * area)[k].sum(),
                       np.abs(s_rp - rp)[k].max() * vol / (np.abs(rp) * area)[k].sum())
    assert polar_err == pytest.approx(expect_polar, rel=1e-8)
    # sigmaError with zero reference stresses: each component's largest
    # magnitude over its signed area-weighted mean, the largest of the three.
    # Only the sxx term is well conditioned here: with no y traction and the
    # plate symmetric about both axes, the area integrals of syy and tau are
    # zero up to round-off, so their terms are round-off ratios of any size
    # and sign. The result is at least the sxx term and finite.
    vol = area.sum()
    expect_sxx = np.abs(sxx).max() * vol / (sxx * area).sum()
    assert np.isfinite(cart_err)
    assert cart_err >= expect_sxx * (1 - 1e-8)
    # the polar-coordinate VTK: strains from the tensor shear gamma / 2
    v = vtk.read_solution_vtk(out)["cell_fields"]
    for name, ref in zip(("Sigma_rr", "Sigma_phiphi", "Tau_rphi"), (rr, pp, rp)):
        assert rel_l2(v[name], ref) < 1e-8, name
    err, epp, erp = _polar(c, o["exx"], o["eyy"], 0.5 * o["gamma"])
    for name, ref in zip(("Eps_rr", "Eps_phiphi", "Gamma_rphi"), (err, epp, erp)):
        assert rel_l2(v[name], ref) < 1e-8, name
    assert "Sigma_xx" not in v
