"""The allocation-free secant update (cp_secant_update_noalloc) against the
regular entry point (cp_secant_update) on the same state, two calls in a row.

It exists for callers that cannot allocate device memory (a framework whose
caching allocator owns the device memory, loops with a fixed memory budget):
the caller passes device buffers it owns, here torch tensors, and the
library's only scratch is a static device array. This file is collected last
on purpose, so that a run stopping at its first failure has already run every
other test."""
import ctypes
import os

import numpy as np
import pytest

import cudaplasticity_b200 as cp
import product_runner
import scenarios
from cudaplasticity_b200 import _capi

pytestmark = pytest.mark.gpu

FIELDS = ["exx", "eyy", "gamma", "eps_i", "sxx", "syy", "tau", "sig_i", "table_s"]


def test_noalloc_update_matches_regular_update(workdir):
    import torch

    ctx = cp.Context(0)
    torch.cuda.set_device(0)
    m, lines = scenarios.scenario_lines("hole12_pow", os.path.join(workdir, "m.bin"))
    job, (rp, mask, uv) = product_runner.build_inputs(lines, m)
    mat = product_runner.material_of(job)
    inst = cp.Instance(ctx, m, mat)
    inst.set_loads(rp, mask, uv)
    inst.assemble()
    inst.cg_solve(1e-12)

    dev = torch.device("cuda:0")
    u = torch.tensor(inst.field("uv"), dtype=torch.float64, device=dev)
    xy = torch.tensor(np.ascontiguousarray(m["node_xy"]).ravel(), dtype=torch.float64, device=dev)
    e4 = torch.tensor(np.ascontiguousarray(m["elem4"]).ravel(), dtype=torch.int32, device=dev)
    ne = m["elem4"].shape[0]
    E_c = torch.tensor(inst.field("E_c"), dtype=torch.float64, device=dev)
    nu_c = torch.tensor(inst.field("nu_c"), dtype=torch.float64, device=dev)
    psi = torch.zeros(ne, dtype=torch.float64, device=dev)
    fields = torch.zeros(9 * ne, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()

    for call in range(2):
        err = ctypes.c_double()
        st = _capi.lib().cp_secant_update_noalloc(
            None, ctypes.byref(mat), m["node_xy"].shape[0], xy.data_ptr(), ne, e4.data_ptr(), u.data_ptr(),
            E_c.data_ptr(), nu_c.data_ptr(), psi.data_ptr(), fields.data_ptr(), ctypes.byref(err))
        assert st == 0, cp._capi.lib().cp_status_string(st)
        ref_err = inst.secant_update()
        assert err.value == pytest.approx(ref_err, rel=1e-12, abs=0.0), call
        f = fields.cpu().numpy().reshape(9, ne)
        for k, name in enumerate(FIELDS):
            ref = inst.field(name)
            scale = max(np.linalg.norm(ref), 1e-300)
            assert np.linalg.norm(f[k] - ref) / scale <= 1e-12, (call, name)
        for name, t in (("E_c", E_c), ("nu_c", nu_c), ("psi", psi)):
            ref = inst.field(name)
            assert np.linalg.norm(t.cpu().numpy() - ref) / np.linalg.norm(ref) <= 1e-12, (call, name)

    # sizes beyond the stated maximum are refused before any work
    err = ctypes.c_double()
    st = _capi.lib().cp_secant_update_noalloc(None, ctypes.byref(mat), m["node_xy"].shape[0], xy.data_ptr(),
                                              1_048_577, e4.data_ptr(), u.data_ptr(), E_c.data_ptr(), nu_c.data_ptr(),
                                              psi.data_ptr(), fields.data_ptr(), ctypes.byref(err))
    assert st == _capi.CP_ERR_INVALID
    inst.close()
    ctx.close()
