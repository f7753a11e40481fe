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
