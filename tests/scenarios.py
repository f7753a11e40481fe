"""Parity scenarios shared by the golden-fixture script, the oracle pins and
the GPU parity tests. Each scenario is a mesh plus the lines of a job in the
harness syntax (material, diagram, loads). Units are those of the scenario
(the configuration-style ones use mm and MPa).

Scenarios with ``reference=True`` contain only what the reference supports
(Q4 and Q8 elements, its BC types) and have golden fixtures made by running
the reference. The 8-node meshes come from the product's host generators,
which are pinned to the reference's own (order 2, Mesh::remapOrder) by the
digests in golden/ref_meshes.json.
"""
import numpy as np

import meshgen

E304, NU304 = 193000.0, 0.29
TIGHT = ["cg_eps 1e-13", "outer_eps 1e-12", "max_outer 400"]

# five-segment piecewise-linear diagram: elastic to (sy/E, sy), then tangent
# slopes 20 GPa .. 0.5 GPa (geometric), segment widths 1e-3
def piecewise_lines(E, sy, slopes=(20000.0, 7952.7, 3162.3, 1257.4, 500.0), width=1e-3):
    pts = [(sy / E, sy)]
    for h in slopes:
        e, s = pts[-1]
        pts.append((e + width, s + h * width))
    flat = " ".join(f"{e!r} {s!r}" for e, s in pts)
    return f"diagram piecewise {E!r} {len(pts)} {flat}"


def _hole12():
    return meshgen.hole_plate(-3.0, 3.0, -2.0, 2.0, 0.5, 12, 8)


def _ogrid(n_c4, rad_n):
    return meshgen.hole_plate(-100.0, 100.0, -100.0, 100.0, 20.0, n_c4, n_c4, rad_n=rad_n)


def _ring():
    return meshgen.ring(50.0, 100.0, 32, 8)


def _q8(make):
    """An 8-node mesh from the host generators, with its second-order nodes."""
    def build():
        import cudaplasticity_b200 as cp

        m = make(cp).arrays()
        sec = np.zeros(len(m["node_xy"]), np.uint8)
        sec[np.asarray(m["elem8"])[:, 4:].ravel()] = 1
        m["sec_ord"] = sec
        return m
    return build


_PT_LOADS = ["force 1 170 0 0", "force 3 -170 0 0", "fixvertaxis 0", "fixhoraxis 0"]
_OGRID_LOADS = ["force 2 0 200 0", "fixborderhor 0", "fixpoint -100 -100"]


def _ring_lines(mesh):
    return ["force 0 200 0 1"] + [f"fixdof {d}" for d in meshgen.axis_dofs(mesh["node_xy"])]


SCENARIOS = {
    # plasticityTest material (src/Main.cpp:252-296) on a 320-element plate
    "hole12_pow": dict(mesh=_hole12, reference=True,
                       lines=[f"diagram power {E304} 170 1930 0.015", f"material {E304} {NU304} 1"] + _PT_LOADS),
    # aitken_plast1 material: linear hardening K_T = 0.1 E
    "hole12_lin": dict(mesh=_hole12, reference=True,
                       lines=[f"diagram linear {E304} 170 19300", f"material {E304} {NU304} 1"] + _PT_LOADS),
    "hole12_strain": dict(mesh=_hole12, reference=True,
                          lines=[f"diagram linear {E304} 170 19300", f"material {E304} {NU304} 1", "plane strain"] + _PT_LOADS),
    # hole-plate O-grid (16 circumferential x 8 radial), bilinear
    # sy = 250, Et = 2 GPa, top traction 200 MPa in 10 increments
    "ogrid16_bilin": dict(mesh=lambda: _ogrid(4, 8), reference=True, levels=10,
                          lines=["diagram linear 210000 250 2000", "material 210000 0.3 1"] + _OGRID_LOADS),
    # Hollomon hardening sy (1 + ep/e0)^n, 4 increments to 220 MPa
    "ogrid16_hollomon": dict(mesh=lambda: _ogrid(4, 8), reference=True, levels=4,
                             lines=["diagram hollomon 210000 250 0.002 0.2", "material 210000 0.3 1",
                                    "force 2 0 220 0", "fixborderhor 0", "fixpoint -100 -100"]),
    # ring under internal pressure, piecewise diagram (as in the request streams)
    "ring_pw": dict(mesh=_ring, reference=True, lines_fn=lambda m: [piecewise_lines(210000.0, 300.0), "material 210000 0.3 1"] + _ring_lines(m)),
    # solverTest (src/Main.cpp:14-38): elastic 4x4 patch
    "rect_elastic": dict(mesh=lambda: meshgen.rect(-1.0, 1.0, -1.0, 1.0, 4, 4), reference=True, mode="elastic",
                         lines=[f"diagram linear {E304} 170000000 {E304}", f"material {E304} {NU304 * 1e-6!r} 1",
                                "displ 2 0 0 0 1", "force 0 1 0 0"]),
    # 8-node elements (Q8, 3x3 Gauss points): the plasticityTest plate ...
    "hole12_q8_pow": dict(mesh=_q8(lambda cp: cp.Mesh.rect_with_hole(-3.0, 3.0, -2.0, 2.0, 0.5, 12, 8, order=2)),
                          reference=True,
                          lines=[f"diagram power {E304} 170 1930 0.015", f"material {E304} {NU304} 1"] + _PT_LOADS),
    # ... the O-grid with a bilinear diagram in 5 increments and gravity ...
    "ogrid8_q8_bilin": dict(mesh=_q8(lambda cp: cp.Mesh.rect_with_hole(-100.0, 100.0, -100.0, 100.0, 20.0, 2, 2,
                                                                        rad_n=4, order=2)),
                            reference=True, levels=5,
                            lines=["diagram linear 210000 250 2000", "material 210000 0.3 1", "gravity 9.81 0 -1"]
                            + _OGRID_LOADS),
    # ... and the ring under internal pressure (quadratic edges turned with
    # the curved border), piecewise diagram
    "ring_q8_pw": dict(mesh=_q8(lambda cp: cp.Mesh.ring(50.0, 100.0, 16, 4, order=2)), reference=True,
                       lines_fn=lambda m: [piecewise_lines(210000.0, 300.0), "material 210000 0.3 1"] + _ring_lines(m)),
    # Parity at configuration size (state-only fixtures, see STATE_FIELDS):
    # the benchmark's own job, the 64x64 O-grid plate (4160 nodes, 8320 DOF),
    # bilinear sy = 250, Et = 2 GPa, 200 MPa in 10 increments ...
    "config1_bilin": dict(mesh=lambda: _ogrid(16, 64), state_fixture=True, levels=10,
                          lines=["max_outer 5000", "diagram linear 210000 250 2000", "material 210000 0.3 1"]
                          + _OGRID_LOADS),
    # ... and a 128 x 64 O-grid (8320 nodes: more than one thread-block
    # cluster holds, so the FP64 solve takes the grid-wide form), Hollomon
    # hardening, 4 increments to 220 MPa
    "ogrid128x64_hollomon": dict(mesh=lambda: _ogrid(32, 64), state_fixture=True, levels=4,
                                 lines=["max_outer 5000", "diagram hollomon 210000 250 0.002 0.2",
                                        "material 210000 0.3 1",
                                        "force 2 0 220 0", "fixborderhor 0", "fixpoint -100 -100"]),
    # CST extension (no reference counterpart): the hole-plate O-grid split
    "ogrid16_t3": dict(mesh=lambda: meshgen.split_t3(_ogrid(4, 8)), reference=False, levels=10,
                       lines=["diagram linear 210000 250 2000", "material 210000 0.3 1"] + _OGRID_LOADS),
}


# fields kept in the state-only fixtures of the configuration-size scenarios
STATE_FIELDS = ["uv", "eps_i", "sig_i", "psi", "eps_p_i"]


def scenario_lines(name, mesh_path, mode=None, extra=()):
    sc = SCENARIOS[name]
    m = sc["mesh"]()
    lines = list(sc.get("lines", [])) + (sc["lines_fn"](m) if "lines_fn" in sc else [])
    lines = [f"mode {mode or sc.get('mode', 'phases')}", f"mesh file {mesh_path}",
             f"levels {sc.get('levels', 1)}"] + TIGHT + lines + list(extra)
    return m, lines


def mesh_digest(m):
    import hashlib

    h = hashlib.sha256()
    for k in ("node_xy", "elem3", "elem4"):
        h.update(np.ascontiguousarray(np.asarray(m[k], dtype=np.float64 if k == "node_xy" else np.int32)).tobytes())
    for b in m["borders"]:
        h.update(np.asarray(b, dtype=np.int32).tobytes())
    e8 = np.asarray(m.get("elem8", ()), dtype=np.int32)
    if e8.size:  # 8-node meshes only: the digests of 4-node meshes are unchanged
        h.update(b"elem8")
        h.update(np.ascontiguousarray(e8).tobytes())
        h.update(np.ascontiguousarray(np.asarray(m["sec_ord"], dtype=np.uint8)).tobytes())
    return h.hexdigest()
