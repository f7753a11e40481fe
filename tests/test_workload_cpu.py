"""The seeded request generator of the batched and served workloads
(cudaplasticity_b200/workload.py), CPU only: every request is reproducible
alone from (base seed, index), and the drawn parameters stay inside the
ranges the workload specifies (plates and rings alternating, DOF log-uniform
in [dof_min, dof_max], a monotone five-segment hardening diagram with slopes
20 GPa down to 0.5 GPa, Dirichlet masks that remove the rigid-body modes)."""
import numpy as np
import pytest

from cudaplasticity_b200 import workload


def test_requests_are_reproducible_alone():
    a = workload.instance(7, seed=123, dof_min=2000, dof_max=6000, increments=(5, 12))
    workload.instance(3, seed=123)  # another draw in between changes nothing
    b = workload.instance(7, seed=123, dof_min=2000, dof_max=6000, increments=(5, 12))
    assert a["params"] == b["params"]
    for k in ("node_xy", "elem4"):
        assert np.array_equal(a["mesh"][k], b["mesh"][k])
    for k in ("rp", "mask", "uv"):
        assert np.array_equal(a[k], b[k])
    assert a["levels"] == b["levels"] and 5 <= a["levels"] <= 12


@pytest.mark.parametrize("i", range(12))
def test_request_parameters_stay_in_their_ranges(i):
    w = workload.instance(i, seed=20261203, dof_min=2000, dof_max=20000)
    p = w["params"]
    assert p["kind"] == ("plate" if i % 2 == 0 else "ring")
    if p["kind"] == "plate":
        assert 10.0 <= p["hole_radius"] <= 60.0 and 100.0 <= p["traction"] <= 300.0
    else:
        assert 80.0 <= p["outer_radius"] <= 150.0 and 100.0 <= p["pressure"] <= 300.0
    assert p["n_c"] % 4 == 0
    # the mesh size tracks the drawn DOF count (O-grid rounding aside)
    assert 1000 <= p["dof"] <= 30000
    assert p["dof"] == 2 * w["mesh"]["node_xy"].shape[0]
    # monotone diagram: yield point on the elastic line, then decreasing slopes
    pts = np.array(p["points"])
    assert len(pts) == 6 and 200.0 <= p["sigma_y"] <= 400.0
    assert abs(pts[0, 1] - workload.E_MPA * pts[0, 0]) <= 1e-9 * pts[0, 1]
    slopes = np.diff(pts[:, 1]) / np.diff(pts[:, 0])
    assert np.allclose(slopes, workload.SLOPES, rtol=1e-9)
    assert np.all(np.diff(slopes) < 0) and np.all(np.diff(pts[:, 0]) > 0)
    # Dirichlet set: DOFs fixed in both directions; a nonzero load
    mask = np.asarray(w["mask"]).reshape(-1, 2)
    assert mask[:, 0].min() == 0 and mask[:, 1].min() == 0
    assert np.abs(w["rp"]).sum() > 0


def test_dof_draws_are_log_uniform():
    """Over many indices the drawn DOF counts spread over the whole range in
    log space (quartiles near the log-uniform ones)."""
    d = np.array([workload.instance(i, seed=99, dof_min=2000, dof_max=200000)["params"]["dof"]
                  for i in range(0, 64)])
    q = np.quantile(np.log(d), [0.25, 0.5, 0.75])
    lo, hi = np.log(2000), np.log(200000)
    want = lo + (hi - lo) * np.array([0.25, 0.5, 0.75])
    assert np.all(np.abs(q - want) < 0.2 * (hi - lo))
