"""The drop-in ``solve_batch`` service (contract of the reference's
``TemporalGpuLPBackend`` / ``RepeatedCpuLP``) on the GPU."""
import numpy as np
import pytest

from co_cultivation_metabolic_atlas_b200 import synthetic as syn
from co_cultivation_metabolic_atlas_b200.problem import request
from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="CUDA device required")]


def requests_for(model, lower, upper):
    return [request((model.S, np.zeros(model.S.shape[0]), lower[i], upper[i], model.cost,
                     model.S.shape[0])) for i in range(len(lower))]


def test_rows_match_highs_without_cpu_optimizer(golden_dir, forbid_cpu_optimizers):
    from co_cultivation_metabolic_atlas_b200 import B200LPBackend
    g = np.load(golden_dir / "highs_single.npz")
    model, lower, upper = syn.single_species_workload(8)
    be = B200LPBackend(mode="cold")
    rows = be.solve_batch(requests_for(model, lower, upper), environment_ids=list(range(100, 108)))
    assert all(r.success for r in rows)
    for r, fun in zip(rows, g["fun"]):
        assert abs(r.fun - fun) <= 1e-6 * max(1.0, abs(fun))
        assert r.x.shape == (2600,) and r.y.shape == (1200,)
        assert r.diagnostics["certificate_passed"] and r.diagnostics["cpu_lp_calls"] == 0
    assert be.history[-1]["cpu_lp_calls"] == 0 and be.history[-1]["accepted"] == 8
    be.close()


def test_previous_mode_reuses_certified_solutions():
    from co_cultivation_metabolic_atlas_b200 import B200LPBackend
    model, lower, upper = syn.single_species_workload(4, m=300, n=650)
    reqs = requests_for(model, lower, upper)
    be = B200LPBackend(mode="previous", precision="fp64")
    first = be.solve_batch(reqs, environment_ids=["a", "b", "c", "d"])
    assert all(r.success for r in first)
    again = be.solve_batch(reqs, environment_ids=["a", "b", "c", "d"])
    assert all(r.success for r in again)
    assert all(r.diagnostics["iterations"] == 0 for r in again)
    be.reset(["a"])
    third = be.solve_batch(reqs, environment_ids=["a", "b", "c", "d"])
    assert third[0].diagnostics["iterations"] > 0 and third[1].diagnostics["iterations"] == 0
    be.close()


def test_invalid_requests_fail_before_any_state_change():
    from co_cultivation_metabolic_atlas_b200 import B200LPBackend
    model, lower, upper = syn.single_species_workload(2, m=120, n=260)
    reqs = requests_for(model, lower, upper)
    be = B200LPBackend(mode="previous")
    be.solve_batch(reqs, environment_ids=[1, 2])
    state = dict(be.last_certified)
    history = len(be.history)
    bad = list(reqs)
    c, kw = bad[1]
    kw = dict(kw)
    kw["bounds"] = np.column_stack([upper[1], lower[1]])  # lower > upper
    bad[1] = (c, kw)
    with pytest.raises(ValueError):
        be.solve_batch(bad, environment_ids=[1, 2])
    with pytest.raises(ValueError):
        be.solve_batch(reqs, environment_ids=[1, 1])
    with pytest.raises(ValueError):
        be.solve_batch([], environment_ids=[])
    assert len(be.history) == history and be.last_certified.keys() == state.keys()
    be.close()


def test_unsolved_rows_fail_closed():
    from co_cultivation_metabolic_atlas_b200 import B200LPBackend
    model, lower, upper = syn.single_species_workload(2, m=120, n=260)
    be = B200LPBackend(mode="cold", precision="fp64", iterations=64, fp32_iterations=0, retry_iterations=0)
    rows = be.solve_batch(requests_for(model, lower, upper))
    assert not any(r.success for r in rows)
    assert all(r.x is None and r.fun is None for r in rows)
    assert "no CPU fallback" in rows[0].message
    be.close()
    # by default the rows stopped by the cap continue in a second GPU pass
    be = B200LPBackend(mode="cold", precision="fp64", iterations=64, fp32_iterations=0)
    rows = be.solve_batch(requests_for(model, lower, upper))
    assert all(r.success for r in rows)
    assert be.history[-1]["retried"] == [0, 1] and be.history[-1]["cpu_lp_calls"] == 0
    be.close()


def test_reference_traces_replay_through_the_backend(golden_dir, tmp_path, forbid_cpu_optimizers):
    """LP traces written by the reference's trace writer (one with an
    inequality row) replay through ``solve_batch`` to their HiGHS optima."""
    import shutil
    from co_cultivation_metabolic_atlas_b200 import B200LPBackend, lp_trace
    d = tmp_path / "traces"
    shutil.copytree(golden_dir / "traces", d)
    be = B200LPBackend(mode="cold")
    rows, ref = lp_trace.replay(d, be)
    be.close()
    assert len(rows) == 3
    for r, fun in zip(rows, ref):
        assert r.success, r.message
        assert abs(r.fun - fun) <= 1e-6 * max(1.0, abs(fun))


def test_equality_reduction_presolve_certifies_the_original_lps(golden_dir, forbid_cpu_optimizers):
    """With the exact homogeneous-equality presolve the GPU solves the
    reduced LPs; expanded primals and lifted duals pass the ORIGINAL LPs'
    certificate and reach HiGHS's objectives; a second call warm-starts from
    the compressed previous solutions."""
    from co_cultivation_metabolic_atlas_b200 import B200LPBackend
    from oracle import dfba
    g = np.load(golden_dir / "highs_community.npz")
    models = syn.community_models()
    medium, biomass = syn.initial_environments(4)
    reqs, funs = [], []
    for s, mdl in enumerate(models):
        lo = dfba.uptake_lower_bounds(mdl, medium, biomass, 0.05)
        for e in range(2):
            reqs.append(request((mdl.S, np.zeros(mdl.S.shape[0]), lo[e], mdl.upper, mdl.cost, mdl.S.shape[0])))
            funs.append(float(g[f"s{s}_fun"][e]))
    be = B200LPBackend(mode="previous", equality_reduction=True)
    rows = be.solve_batch(reqs, environment_ids=list(range(6)))
    assert all(r.success for r in rows), [r.message for r in rows]
    for r, fun, (c, kw) in zip(rows, funs, reqs):
        assert abs(r.fun - fun) <= 1e-6 * max(1.0, abs(fun))
        assert r.diagnostics["equality_reduction"] and r.diagnostics["certificate_passed"]
        assert r.x.shape == (kw["A_eq"].shape[1],) and r.y.shape == (kw["A_eq"].shape[0],)
    again = be.solve_batch(reqs, environment_ids=list(range(6)))
    assert all(r.success for r in again)
    assert sum(r.diagnostics["iterations"] for r in again) < sum(r.diagnostics["iterations"] for r in rows)
    be.close()
