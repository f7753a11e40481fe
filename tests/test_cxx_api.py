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
