"""Seeded synthetic problem instances for the batched and served workloads.

Instance i of a stream with base seed S draws everything from its own
generator (seed S + i, through numpy's PCG64), so any instance can be
regenerated alone:

* even i: square plate 200 x 200 mm with a centred hole, radius ~ U[10, 60] mm,
  O-grid of n_c circumferential x n_r radial quads; uniform traction ~ U[100,
  300] MPa on the top edge; bottom edge fixed in y, bottom-left corner fixed;
* odd i: thick ring, inner radius 50 mm, outer ~ U[80, 150] mm, internal
  pressure ~ U[100, 300] MPa (normal traction on the inner border); u_y = 0 on
  the x axis and u_x = 0 on the y axis (symmetry; removes rigid-body modes);
* DOF ~ log-uniform in [dof_min, dof_max]; n_c = n_r ~ sqrt(DOF / 2), n_c a
  multiple of 4 (so that nodes lie on the axes / corners);
* material E = 210 GPa, nu = 0.3, plane stress, h = 1 mm; a 5-segment
  monotone piecewise-linear hardening diagram: sigma_y ~ U[200, 400] MPa, then
  tangent slopes 20 GPa .. 0.5 GPa (geometric), segment widths ~ U[0.5, 2] x
  1e-3 strain, the last segment extending.
Units: mm, N, MPa.
"""
import math

import numpy as np

from . import CP_PLANE_STRESS, Loads, Mesh, material

E_MPA = 210000.0
NU = 0.3
SLOPES = [20000.0 * (500.0 / 20000.0) ** (k / 4.0) for k in range(5)]


def _grid_for(dof):
    n = int(round(math.sqrt(dof / 2.0)))
    n_c = max(8, 4 * int(round(n / 4.0)))
    n_r = max(4, int(round(dof / 2.0 / n_c)) - 1)
    return n_c, n_r


def instance(i, seed=20261203, dof_min=2000, dof_max=200000, increments=None):
    """Returns a dict: kind, params, mesh arrays, material, rp, mask, uv,
    levels (load increments; 1 unless ``increments`` is a (lo, hi) range)."""
    rng = np.random.default_rng(seed + i)
    dof = math.exp(rng.uniform(math.log(dof_min), math.log(dof_max)))
    n_c, n_r = _grid_for(dof)
    sy = rng.uniform(200.0, 400.0)
    widths = rng.uniform(0.5e-3, 2e-3, size=5)
    pts = [(sy / E_MPA, sy)]
    for h, w in zip(SLOPES, widths):
        e, s = pts[-1]
        pts.append((e + w, s + h * w))
    mat = material(E_MPA, NU, h=1.0, plane=CP_PLANE_STRESS, diagram="piecewise", points=pts)
    L = Loads()
    if i % 2 == 0:
        R = rng.uniform(10.0, 60.0)
        traction = rng.uniform(100.0, 300.0)
        mesh = Mesh.rect_with_hole(-100.0, 100.0, -100.0, 100.0, R, n_c // 4, n_c // 4, rad_n=n_r)
        L.set_force(2, 0.0, traction).fix_border_hor(0).fix_point(-100.0, -100.0)
        params = dict(kind="plate", hole_radius=R, traction=traction)
    else:
        b = rng.uniform(80.0, 150.0)
        p = rng.uniform(100.0, 300.0)
        mesh = Mesh.ring(50.0, b, n_c, n_r)
        L.set_force(0, p, 0.0, True)
        xy = mesh.arrays()["node_xy"]
        r = np.hypot(xy[:, 0], xy[:, 1])
        for nd in np.where(np.abs(xy[:, 1]) <= 1e-9 * r)[0]:
            L.fix_dof(2 * int(nd) + 1)
        for nd in np.where(np.abs(xy[:, 0]) <= 1e-9 * r)[0]:
            L.fix_dof(2 * int(nd))
        params = dict(kind="ring", outer_radius=b, pressure=p)
    arrays = mesh.arrays()
    rp, mask, uv = L.build(mesh, h=1.0)
    levels = 1
    if increments is not None:
        levels = int(rng.integers(increments[0], increments[1] + 1))
    params.update(index=i, seed=seed + i, n_c=n_c, n_r=n_r, dof=2 * arrays["node_xy"].shape[0],
                  sigma_y=sy, points=pts, levels=levels)
    return dict(params=params, mesh=arrays, material=mat, rp=rp, mask=mask, uv=uv, levels=levels)
