"""CPU tests of the product's boundary and host logic (no GPU compute):
the C ABI library loads and exports every declared symbol; the host-side
drop-in classes (mesh generators, load/BC builder) reproduce the reference
bit for bit; device entry points fail cleanly without a device."""
import glob
import json
import os
import re

import numpy as np
import pytest

import cudaplasticity_b200 as cp
import meshgen
import scenarios
from cudaplasticity_b200 import _capi
from conftest import ROOT, have_gpu

import product_runner


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        names += re.findall(r"CP_API\s+[\w\s\*]+?\b(\w+)\s*\(", txt)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = _capi.lib()
    names = declared_functions()
    assert len(names) >= 40
    for n in names:
        assert hasattr(lib, n), n
    # and the ctypes table covers all of them
    assert set(names) == set(_capi.declared_symbols())


def test_version_and_status_strings():
    assert "sm_100a" in cp.version()
    assert _capi.lib().cp_status_string(4).decode() == "iteration limit reached"


def _digest_of(m):
    a = m.arrays()
    d = dict(node_xy=a["node_xy"], elem3=a["elem3"], elem4=a["elem4"], borders=a["borders"])
    if "elem8" in a:  # second-order nodes: the mid-side nodes of the 8-node elements
        sec = np.zeros(len(a["node_xy"]), np.uint8)
        sec[a["elem8"][:, 4:].ravel()] = 1
        d.update(elem8=a["elem8"], sec_ord=sec)
    return scenarios.mesh_digest(d)


def test_product_mesh_generators_match_reference(golden_dir):
    ref = json.load(open(os.path.join(golden_dir, "ref_meshes.json")))
    makers = {
        "hole -3 3 -2 2 0.5 48 32 1": lambda: cp.Mesh.rect_with_hole(-3, 3, -2, 2, 0.5, 48, 32),
        "hole -3 3 -2 2 0.5 12 8 1": lambda: cp.Mesh.rect_with_hole(-3, 3, -2, 2, 0.5, 12, 8),
        "hole -100 100 -100 100 20 16 16 1": lambda: cp.Mesh.rect_with_hole(-100, 100, -100, 100, 20, 16, 16),
        "ring 50 120 32 8 1": lambda: cp.Mesh.ring(50, 120, 32, 8),
        "ring 0.1 0.2 40 5 1": lambda: cp.Mesh.ring(0.1, 0.2, 40, 5),
        "rect -1 1 -1 1 4 4 1": lambda: cp.Mesh.rect(-1, 1, -1, 1, 4, 4),
        "rect -3 3 -2 2 6 4 1": lambda: cp.Mesh.rect(-3, 3, -2, 2, 6, 4),
        # 8-node meshes (Mesh::remapOrder)
        "hole -3 3 -2 2 0.5 12 8 2": lambda: cp.Mesh.rect_with_hole(-3, 3, -2, 2, 0.5, 12, 8, order=2),
        "ring 50 120 16 4 2": lambda: cp.Mesh.ring(50, 120, 16, 4, order=2),
        "rect -3 3 -2 2 6 4 2": lambda: cp.Mesh.rect(-3, 3, -2, 2, 6, 4, order=2),
    }
    for spec, mk in makers.items():
        m = mk()
        assert _digest_of(m) == ref[spec]["digest"], spec
        assert m.max_index_diff() == ref[spec]["max_index_diff"], spec


@pytest.mark.parametrize("name", ["hole_renum11", "ring_q8_renum", "ogrid_smooth", "rect_renum_ties"])
def test_mesh_tooling_matches_reference(name, golden_dir):
    """Mesh::renumByDirection (ties in the reference's merge order),
    smoothRing, aspectRatio, skewAngleSin and avrElemSize of the drop-in Mesh
    against the reference's own, on the meshes of its generators: the
    renumbered / smoothed mesh bit for bit (digest), the quality figures bit
    for bit."""
    import sys

    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_golden import MESH_TOOLS

    g = dict(np.load(os.path.join(golden_dir, "ref_mesh_tools.npz")))
    spec, ops = MESH_TOOLS[name]
    w = spec.split()
    f = [float(x) for x in w[1:]]
    if w[0] == "hole":
        mesh = cp.Mesh.rect_with_hole(*f[:5], int(f[5]), int(f[6]), order=int(f[7]))
    elif w[0] == "ring":
        mesh = cp.Mesh.ring(f[0], f[1], int(f[2]), int(f[3]), order=int(f[4]))
    else:
        mesh = cp.Mesh.rect(*f[:4], int(f[4]), int(f[5]), order=int(f[6]))
    for op in ops:
        if op[0] == "renum":
            mesh.renum_by_direction(op[1], op[2])
        else:
            mesh.smooth_ring(op[1])
    assert _digest_of(mesh) == str(g[f"{name}_digest"])
    q = mesh.quality()
    assert np.array_equal(q["aspect"], g[f"{name}_aspect"])
    assert np.array_equal(q["skew_sin"], g[f"{name}_skew_sin"])
    assert q["avr_elem_size"] == float(g[f"{name}_avr_elem_size"][0])


def test_product_ogrid_matches_test_generator():
    """The O-grid with a free radial count (benchmark meshes) and the T3 split."""
    a = cp.Mesh.rect_with_hole(-100, 100, -100, 100, 20, 16, 16, rad_n=64).arrays()
    b = meshgen.hole_plate(-100, 100, -100, 100, 20, 16, 16, rad_n=64)
    assert np.array_equal(a["node_xy"], b["node_xy"]) and np.array_equal(a["elem4"], b["elem4"])
    t = cp.Mesh.rect_with_hole(-100, 100, -100, 100, 20, 4, 4, rad_n=8).split_t3().arrays()
    tb = meshgen.split_t3(meshgen.hole_plate(-100, 100, -100, 100, 20, 4, 4, rad_n=8))
    assert np.array_equal(t["elem3"], tb["elem3"]) and t["elem4"].size == 0


@pytest.mark.parametrize("name", [n for n, s in scenarios.SCENARIOS.items() if s.get("reference")])
def test_product_loads_match_reference(name, golden_dir, workdir):
    """initConditions restated in the C++ drop-in classes: the right-hand side
    and the Dirichlet mask equal the reference's bit for bit."""
    g = np.load(os.path.join(golden_dir, f"{name}.npz"))
    m, lines = scenarios.scenario_lines(name, os.path.join(workdir, "m.bin"))
    _, (rp, mask, uv) = product_runner.build_inputs(lines, m)
    assert np.array_equal(mask, g["mask"])
    assert np.array_equal(rp, g["rp"])


def test_loads_reject_bad_border():
    m = cp.Mesh.rect(0, 1, 0, 1, 2, 2)
    with pytest.raises(cp.CuplastError):
        cp.Loads().set_force(9, 1.0, 0.0).build(m)


def test_footprint_is_host_only():
    m = meshgen.hole_plate(-100, 100, -100, 100, 20, 16, 16, rad_n=64)
    f64 = cp.footprint(m, cp.CP_PREC_FP64)
    fmx = cp.footprint(m, cp.CP_PREC_MIXED)
    assert fmx > f64 > 4160 * 36 * 8


@pytest.mark.skipif(have_gpu(), reason="checks the no-device path")
def test_device_calls_fail_cleanly_without_gpu():
    assert cp.device_count() == 0
    with pytest.raises(cp.CuplastError) as e:
        cp.Context(0)
    assert e.value.status == _capi.CP_ERR_NO_DEVICE


@pytest.mark.parametrize("name", ["mixed", "quirks"])
def test_inp_loader_matches_reference(name, golden_dir):
    """Mesh::loadFromFile (src/Mesh.cu:725-937): the product's reader gives
    the arrays the reference's own reader made of the same file, bit for bit
    (fixtures from tests/golden/make_golden.py). ``quirks`` covers the
    reference's rule that a block's terminating line is consumed with it."""
    g = dict(np.load(os.path.join(golden_dir, f"inp_{name}.npz")))
    a = cp.Mesh.load(os.path.join(golden_dir, f"inp_{name}.inp")).arrays()
    assert np.array_equal(a["node_xy"].ravel(), g["node_xy"])
    assert np.array_equal(a["elem3"].ravel(), g["elem3"])
    assert np.array_equal(a["elem4"].ravel(), g["elem4"])
    assert len(g["elem8"]) == 0
    assert [len(b) for b in a["borders"]] == list(g["border_len"])
    assert np.array_equal(np.concatenate(a["borders"]), g["border_nodes"])


def test_inp_loader_rejects_bad_files(tmp_path):
    with pytest.raises(cp.CuplastError) as e:
        cp.Mesh.load(tmp_path / "mesh.msh")
    assert e.value.status == _capi.CP_ERR_INVALID
    with pytest.raises(cp.CuplastError) as e:
        cp.Mesh.load(tmp_path / "missing.inp")
    assert e.value.status == _capi.CP_ERR_INVALID
    q8 = tmp_path / "q8.inp"
    q8.write_text("*NODE\n" + "".join(f"{i + 1}, {i % 3}.0, {i // 3}.0\n" for i in range(9)) +
                  "**\n*ELEMENT, TYPE=S8R\n1, 1, 3, 9, 7, 2, 6, 8, 4\n")
    m = cp.Mesh.load(q8)  # read into elem8, as the reference's reader does
    assert m.count8() == 1
    assert list(m.arrays()["elem8"][0]) == [0, 2, 8, 6, 1, 5, 7, 3]
    bad = tmp_path / "bad.inp"
    bad.write_text("*NODE\n1, 0.0, 0.0\n2, 1.0, 0.0\n**\n*ELEMENT, TYPE=S3\n1, 1, 2, 9\n")
    with pytest.raises(cp.CuplastError) as e:
        cp.Mesh.load(bad)  # a node that does not exist
    assert e.value.status == _capi.CP_ERR_INVALID


def test_batch_and_server_entry_points_validate_arguments_without_a_device():
    """The batch and server C entry points reject missing handles and bad
    options before touching a device; creating a server without a GPU fails
    with CP_ERR_NO_DEVICE and leaves nothing running."""
    import ctypes

    L = _capi.lib()
    inv = _capi.CP_ERR_INVALID
    bo = _capi.cp_batch_opts()
    L.cp_batch_opts_default(ctypes.byref(bo))
    assert (bo.max_instances, bo.cg_per_trip, bo.elem_per_trip, bo.max_width) == (1024, 16, 3, 16)
    out = _capi.c_p()
    assert L.cp_batch_create(None, ctypes.byref(bo), ctypes.byref(out)) == inv
    assert L.cp_batch_add(None, None, None, None) == inv
    assert L.cp_batch_launch(None, _capi.CP_BATCH_RUN_ALL, 0) == inv
    assert L.cp_batch_wait(None, None, None) == inv
    assert L.cp_batch_run(None, _capi.CP_BATCH_RUN_ALL, 0, None, None) == inv
    n = ctypes.c_int()
    assert L.cp_batch_harvest(None, 1, None, None, None, ctypes.byref(n)) == inv
    assert L.cp_batch_interrupt(None) == inv
    assert L.cp_batch_set_tile(None, 0, 4) == inv
    assert L.cp_batch_get_tile(None, 0, ctypes.byref(n)) == inv
    assert L.cp_batch_autotune(None, None) == inv
    assert L.cp_batch_stats(None, None, None, None) == inv
    assert L.cp_batch_progress(None, 0, None, None, None) == inv
    ms = ctypes.c_double()
    assert L.cp_batch_last_run_ms(None, ctypes.byref(ms)) == inv
    so = _capi.cp_server_opts()
    L.cp_server_opts_default(ctypes.byref(so))
    assert so.max_inflight == 1024 and 0.0 < so.hbm_reserve < 1.0 and so.batch.max_instances == 1024
    assert so.fp64_lanes == 8
    srv = _capi.c_p()
    assert L.cp_server_create(ctypes.byref(so), ctypes.byref(srv)) == _capi.CP_ERR_NO_DEVICE
    assert not srv.value
    so.fp64_lanes = -1
    assert L.cp_server_create(ctypes.byref(so), ctypes.byref(srv)) == inv
    so.fp64_lanes = 8
    so.max_inflight = 0
    assert L.cp_server_create(ctypes.byref(so), ctypes.byref(srv)) == inv
    rid = ctypes.c_longlong()
    assert L.cp_server_submit(None, None, None, None, None, None, None, ctypes.byref(rid)) == inv
    assert L.cp_server_wait(None, 1, 0.0, None, None, None) == inv
    assert L.cp_server_get_stats(None, None) == inv
    assert L.cp_server_destroy(None) == inv
    assert L.cp_secant_update_noalloc(None, None, 0, None, 0, None, None, None, None, None, None, None) == inv
    ms, by = ctypes.c_double(), ctypes.c_double()
    assert L.cp_bench_assemble(None, 0, 1, ctypes.byref(ms), ctypes.byref(by)) == inv
    # host-side mesh tooling validates its arguments
    m = cp.Mesh.rect_with_hole(-3, 3, -2, 2, 0.5, 12, 8)
    assert L.cpx_mesh_smooth_ring(m._h, 7) == inv  # node count not a multiple of the column count
    assert L.cpx_mesh_smooth_ring(m._h, 2) == inv
    assert L.cpx_mesh_renum_by_direction(None, 1.0, 1.0) == inv
    assert L.cpx_mesh_quality(None, None, None, None) == inv


@pytest.mark.parametrize("name", ["hole_q8", "ring_q8", "rect_q8", "rect_points", "ring_mixed"])
def test_q8_and_point_loads_match_reference(name, golden_dir):
    """initConditions (src/PlasticitySolver.cu:812-1005) against the
    reference's own load builder on the same meshes: on 8-node meshes the
    consistent quadratic-edge loads (1/3, 4/3, 1/3 weights, normal pressure
    on curved edges) and 8-node body forces (-1/12 per corner, 1/3 per
    mid-side node); on 4-node meshes point forces, prescribed points, whole
    prescribed borders, one-axis border fixes and a tangential traction
    component. Dirichlet masks and prescribed values bit for bit, forces up
    to the summation order of shared nodes (1e-14 of the largest load)."""
    import sys

    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
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
    assert (mesh.count8() > 0) == (name in Q8_LOADS)
    job = product_runner.parse(lines)
    rp, mask, uv = product_runner.loads_of(job).build(mesh, h=job["h"], rho=1.0)
    ref = g[f"{name}_rp"]
    assert np.max(np.abs(rp - ref)) <= 1e-14 * np.max(np.abs(ref))
    assert np.array_equal(mask, g[f"{name}_mask"])
    assert np.array_equal(uv, g[f"{name}_uv"])
