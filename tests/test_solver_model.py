"""The numpy model of the product's FP64 solve (tests/solver_model.py) on
the benchmark's configuration-1 job: it reproduces the B200's outer and CG
iteration counts to a few per cent, and it is where the recycled initial
guesses (cp_solve_opts.recycle) were found; their effect in the model
matches the one measured on the B200 (40.1k -> 27.4k CG iterations)."""
import numpy as np
import pytest

from solver_model import PlateModel, chol_drop_solve

# measured on the B200 through bench.py's solve (CUDA events, same options)
GPU_PLAIN = (187, 40121)
GPU_RECYCLE6 = (180, 27445)


@pytest.fixture(scope="module")
def model():
    import bench

    _, arrays, _, rp, mask, uv = bench.build_problem()
    return PlateModel(arrays["node_xy"], arrays["elem4"], rp, mask, uv, 210000.0, 0.3, 250.0, 2000.0)


def test_small_solve_drops_dependent_increments():
    rng = np.random.default_rng(3)
    k = rng.standard_normal((20, 20))
    k = k @ k.T + 20 * np.eye(20)
    w = rng.standard_normal((20, 3))
    w = np.column_stack([w, w[:, 0] * 2.0])  # the fourth increment repeats the first
    r0 = rng.standard_normal(20)
    y = chol_drop_solve(w.T @ k @ w, w.T @ r0)
    assert y[3] == 0.0
    # the kept part is the exact Galerkin solution on the independent increments
    w3 = w[:, :3]
    np.testing.assert_allclose(y[:3], np.linalg.solve(w3.T @ k @ w3, w3.T @ r0), rtol=1e-10)


@pytest.mark.slow
def test_model_reproduces_the_gpu_counts_and_the_recycling_gain(model):
    outer0, cg0, u0 = model.solve()
    outer6, cg6, u6 = model.solve(recycle=6)
    assert abs(outer0 - GPU_PLAIN[0]) <= 0.05 * GPU_PLAIN[0]
    assert abs(cg0 - GPU_PLAIN[1]) <= 0.05 * GPU_PLAIN[1]
    assert abs(cg6 - GPU_RECYCLE6[1]) <= 0.05 * GPU_RECYCLE6[1]
    assert cg6 < 0.75 * cg0
    # both stop at outer 1e-6 through different iterates: close, not equal
    assert np.linalg.norm(u6 - u0) / np.linalg.norm(u0) < 1e-4


def test_deflation_model_on_a_small_plate():
    """The deflated variant (a candidate for the cluster CG) on a 16 x 16
    O-grid: the same fixed point within the stop rule, no more CG iterations
    than the recycled initial guesses alone."""
    import cudaplasticity_b200 as cp

    mesh = cp.Mesh.rect_with_hole(-100.0, 100.0, -100.0, 100.0, 20.0, 4, 4, rad_n=16)
    loads = cp.Loads().set_force(2, 0.0, 200.0).fix_border_hor(0).fix_point(-100.0, -100.0)
    rp, mask, uv = loads.build(mesh)
    a = mesh.arrays()
    m = PlateModel(a["node_xy"], a["elem4"], rp, mask, uv, 210000.0, 0.3, 250.0, 2000.0)
    o1, c1, u1 = m.solve(recycle=6)
    o2, c2, u2 = m.solve(recycle=6, deflate=True)
    assert c2 <= c1
    assert np.linalg.norm(u2 - u1) / np.linalg.norm(u1) < 1e-4


def test_library_small_solve_matches_the_model():
    """cpx_recycle_solve runs the device's small solve on the host: it
    agrees with the model's Cholesky-with-drop on random Gram systems, with
    and without dependent increments, for every count 0..6."""
    import ctypes

    from cudaplasticity_b200 import _capi as C

    lib = C.lib()
    rng = np.random.default_rng(11)
    for trial in range(40):
        cnt = trial % 7
        n = 30
        k = rng.standard_normal((n, n))
        k = k @ k.T + n * np.eye(n)
        w = rng.standard_normal((n, max(cnt, 1)))[:, :cnt]
        if cnt >= 3 and trial % 2:
            w[:, 2] = w[:, 0] - 0.5 * w[:, 1]  # a dependent increment
        r0 = rng.standard_normal(n)
        g = w.T @ k @ w
        h = w.T @ r0
        sums = np.zeros(27)
        for kk in range(cnt):
            for j in range(kk + 1):
                sums[kk * (kk + 1) // 2 + j] = g[j, kk]
            sums[21 + kk] = h[kk]
        y = np.zeros(6)
        st = lib.cpx_recycle_solve(sums.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), cnt,
                                   y.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        assert st == 0
        want = chol_drop_solve(g, h) if cnt else np.zeros(0)
        np.testing.assert_allclose(y[:cnt], want, rtol=1e-9, atol=1e-12)
        assert np.all(y[cnt:] == 0.0)
    assert lib.cpx_recycle_solve(None, 1, None) != 0
