"""The allocation-free entry point (fbalp_engine_solve_noalloc).

It serves callers that cannot allocate device memory when they solve
(real-time loops that forbid allocator calls once running, hosts whose device
memory another allocator owns and budgets): after an engine is created up
front, this call uses only the caller's buffers and a fixed library-wide
scratch array.  The test calls it
through the C ABI twice in a row and checks both results against the regular
entry point.  The file name makes pytest collect it last.
"""
import ctypes

import numpy as np
import pytest

from co_cultivation_metabolic_atlas_b200 import synthetic as syn
from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="CUDA device required")]


def _p(t):
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def _noalloc(eng, lower, upper, cost, params, out):
    from co_cultivation_metabolic_atlas_b200 import _native as N
    return eng.lib.fbalp_engine_solve_noalloc(
        eng.handle, eng.count, _p(lower), _p(upper), _p(cost), None, None, None, None, ctypes.byref(params),
        _p(out.status), _p(out.objective), _p(out.x), _p(out.y), _p(out.iterations), _p(out.metrics),
        _p(out.omega))


def test_noalloc_solve_matches_regular_solve_on_two_calls():
    import torch
    from co_cultivation_metabolic_atlas_b200 import _native as N
    from co_cultivation_metabolic_atlas_b200.engine import LPEngine, SolveConfig
    count = 24
    model, lower, upper = syn.single_species_workload(count, m=300, n=650)
    eng = LPEngine([(model.S, 300)])
    lo = torch.as_tensor(lower.ravel(), device="cuda")
    up = torch.as_tensor(upper.ravel(), device="cuda")
    c = torch.as_tensor(np.tile(model.cost, count), device="cuda")
    eng.set_instances(np.zeros(count, np.int32), lo, up, c)
    config = SolveConfig(precision="fp64")
    ref = eng.solve(config=config)
    outs = [eng.allocate_result(), eng.allocate_result()]
    params = config.native()
    torch.cuda.synchronize()
    for out in outs:
        rc = _noalloc(eng, lo, up, c, params, out)
        assert rc == N.FBALP_OK, eng.lib.fbalp_last_error()
    torch.cuda.synchronize()
    # the phase queries cover the regular entry point only
    assert eng.phase_times() == (0.0, 0.0)
    st = ref.status.cpu().numpy()
    assert (st == 0).all()
    for out in outs:
        np.testing.assert_array_equal(out.status.cpu().numpy(), st)
        np.testing.assert_allclose(out.objective.cpu().numpy(), ref.objective.cpu().numpy(), rtol=1e-9, atol=1e-9)
        x, xr = out.x.cpu().numpy(), ref.x.cpu().numpy()
        np.testing.assert_allclose(x, xr, rtol=0, atol=1e-9 * max(1.0, np.abs(xr).max()))
        y, yr = out.y.cpu().numpy(), ref.y.cpu().numpy()
        np.testing.assert_allclose(y, yr, rtol=0, atol=1e-9 * max(1.0, np.abs(yr).max()))
    eng.close()


def test_noalloc_rejects_what_it_cannot_do():
    import torch
    from co_cultivation_metabolic_atlas_b200 import _native as N
    from co_cultivation_metabolic_atlas_b200.engine import LPEngine, SolveConfig
    model, lower, upper = syn.single_species_workload(2, m=120, n=260)
    eng = LPEngine([(model.S, 120)])
    lo = torch.as_tensor(lower.ravel(), device="cuda")
    up = torch.as_tensor(upper.ravel(), device="cuda")
    c = torch.as_tensor(np.tile(model.cost, 2), device="cuda")
    eng.set_instances(np.zeros(2, np.int32), lo, up, c)
    out = eng.allocate_result()
    rc = _noalloc(eng, lo, up, c, SolveConfig(precision="mixed").native(), out)
    assert rc == N.FBALP_ERR_INVALID and b"FP64" in eng.lib.fbalp_last_error()
    # a batch whose metadata alone exceeds the scratch is refused before any work
    params = SolveConfig(precision="fp64").native()
    rc = eng.lib.fbalp_engine_solve_noalloc(eng.handle, 2_000_000, _p(lo), _p(up), _p(c), None, None, None,
                                            None, ctypes.byref(params), _p(out.status), _p(out.objective),
                                            _p(out.x), _p(out.y), _p(out.iterations), _p(out.metrics), None)
    assert rc == N.FBALP_ERR_INVALID and b"scratch" in eng.lib.fbalp_last_error()
    eng.close()
