"""Pin the CPU oracle before trusting it: the reference's own known-answer
LPs, golden certificates produced by the reference's ``_certificate``, and
HiGHS optima of the seeded workloads."""
import json

import numpy as np
import pytest
from scipy.sparse import csr_matrix

from co_cultivation_metabolic_atlas_b200 import synthetic as syn
from oracle import certificate, dfba, highs, pdhg, reference_pdhg


def solve_small(a, rhs, lo, up, c, neq, **kw):
    P = pdhg.prepare(csr_matrix(np.asarray(a, float)), neq)
    return pdhg.solve(P, np.asarray(lo, float), np.asarray(up, float), np.asarray(c, float),
                      np.asarray(rhs, float), check_every=kw.pop("check_every", 8), **kw)


# --- the reference's known-answer tests (tests/test_gpu_pdhg_corrector.py) ---

def test_kat_inequality_dual_sign():
    # :29-42  min -x, x <= 1, 0 <= x <= 2 -> x = 1, HiGHS-style y = -1
    r = solve_small([[1.0]], [1.0], [0.0], [2.0], [-1.0], 0)
    assert r["status"] == pdhg.STATUS_OPTIMAL
    np.testing.assert_allclose(r["x"], [1.0], atol=1e-8)
    np.testing.assert_allclose(r["y"], [-1.0], atol=1e-8)
    cert = certificate.certificate(csr_matrix([[1.0]]), np.array([1.0]), np.array([0.0]),
                                   np.array([2.0]), np.array([-1.0]), 0, r["x"], r["y"])
    assert cert["certificate_passed"]


def test_kat_independent_blocks():
    # :66-82  two independent LPs -> x = [1, 0.5], y = [-1, -1]
    for rhs, want in ((1.0, 1.0), (0.5, 0.5)):
        r = solve_small([[1.0]], [rhs], [0.0], [2.0], [-1.0], 0)
        np.testing.assert_allclose(r["x"], [want], atol=1e-8)
        np.testing.assert_allclose(r["y"], [-1.0], atol=3e-7)


def test_kat_box_only_with_infinite_bound():
    # :85-95  the first variable has no matrix coefficient -> its upper bound
    r = solve_small([[0.0, 1.0]], [0.0], [-np.inf, 0.0], [2.0, np.inf], [-1.0, 0.0], 1)
    assert r["status"] == pdhg.STATUS_OPTIMAL
    np.testing.assert_allclose(r["x"], [2.0, 0.0], atol=1e-10)


def test_kat_infeasible_fails_closed():
    # :98-112  x <= 0 and -x <= -1: never accepted, budget exhausted
    r = solve_small([[1.0], [-1.0]], [0.0, -1.0], [-np.inf], [np.inf], [0.0], 0, max_iters=40,
                    check_every=5)
    assert r["status"] == pdhg.STATUS_ITERATION_LIMIT
    assert r["iterations"] == 40


def test_kat_warm_start_certified_at_iteration_zero():
    # :45-63  warm starts at the optimum are accepted without iterating
    r = solve_small([[1.0]], [2.0], [0.0], [3.0], [1.0], 1, x0=np.array([2.0]),
                    y0=np.array([1.0]), max_iters=0)
    assert pdhg.converged(r["metrics"], 1e-9, 1e-9, 1e-9)


def test_reference_metric_and_primal_weight():
    # :115-120 and :140-164
    a = csr_matrix(np.array([[2.0, -1.0]]))
    tau, sigma = reference_pdhg.metric(a, 0.9)
    np.testing.assert_allclose(sigma, [0.3])
    np.testing.assert_allclose(tau, [0.45, 0.9])
    tau2, sigma2 = reference_pdhg.metric(a, 0.9, primal_weight=2.0)
    np.testing.assert_allclose(sigma2, 2 * sigma)
    np.testing.assert_allclose(tau2, tau / 2)


def test_reference_operator_reaches_kat_optimum():
    x, y = reference_pdhg.iterate(csr_matrix([[1.0]]), np.array([1.0]), np.array([0.0]),
                                  np.array([2.0]), np.array([-1.0]), 0, 200, step_safety=0.9)
    np.testing.assert_allclose(x, [1.0], atol=1e-8)
    np.testing.assert_allclose(y, [-1.0], atol=1e-8)


# --- golden certificates from the reference's _certificate ---

def test_certificate_matches_reference_golden(golden_dir):
    g = np.load(golden_dir / "certificate_golden.npz", allow_pickle=False)
    rows = json.loads(str(g["rows"]))
    model, lower, upper = syn.single_species_workload(4, m=120, n=260)
    a_ineq = csr_matrix(np.array([[1.0, 1.0], [1.0, -1.0], [-1.0, 2.0]]))
    for row in rows:
        key = row["key"]
        x, y = g[f"{key}__x"], g[f"{key}__y"]
        if row["instance"] >= 0:
            i = row["instance"]
            got = certificate.certificate(model.S, np.zeros(model.S.shape[0]), lower[i], upper[i],
                                          model.cost, model.S.shape[0], x, y)
        else:
            got = certificate.certificate(a_ineq, np.array([1.0, 0.5, 2.0]), np.array([0.0, -np.inf]),
                                          np.array([np.inf, 3.0]), np.array([-1.0, -0.5]), 1, x, y)
        for name in ("primal_residual", "dual_violation", "relative_kkt_gap",
                     "bound_complementarity_gap", "row_complementarity_gap"):
            assert got[name] == pytest.approx(row[name], rel=1e-12, abs=1e-15), (key, name)
        assert got["certificate_passed"] == row["certificate_passed"], key


# --- HiGHS and the engine restatement on the seeded workload ---

def test_highs_oracle_reproduces_golden(golden_dir):
    g = np.load(golden_dir / "highs_single.npz")
    model, lower, upper = syn.single_species_workload(8)
    np.testing.assert_array_equal(lower[:, :model.n_exchange], g["exchange_lower"])
    st, fun, x, y = highs.solve_one(model.S, lower[0], upper[0], model.cost)
    assert st == 0 and fun == pytest.approx(float(g["fun"][0]), rel=1e-9)


def test_engine_restatement_matches_highs(golden_dir):
    g = np.load(golden_dir / "highs_single.npz")
    model, lower, upper = syn.single_species_workload(8)
    P = pdhg.prepare(model.S)
    for i in range(2):
        r = pdhg.solve(P, lower[i], upper[i], model.cost)
        assert r["status"] == pdhg.STATUS_OPTIMAL
        fun = float(g["fun"][i])
        assert abs(r["metrics"]["objective"] - fun) <= 1e-6 * max(1.0, abs(fun))
        cert = certificate.certificate(model.S, np.zeros(model.S.shape[0]), lower[i], upper[i],
                                       model.cost, model.S.shape[0], r["x"], r["y"])
        assert cert["certificate_passed"]


def test_mixed_precision_restatement_matches_highs(golden_dir):
    g = np.load(golden_dir / "highs_single.npz")
    model, lower, upper = syn.single_species_workload(8)
    P = pdhg.prepare(model.S)
    r32 = pdhg.solve(P, lower[3], upper[3], model.cost, dtype=np.float32, tol_primal=1e-6,
                     tol_dual=1e-6, tol_gap=1e-4, final_status=pdhg.STATUS_HANDOFF)
    assert r32["status"] == pdhg.STATUS_HANDOFF
    r = pdhg.solve(P, lower[3], upper[3], model.cost, x0=r32["x"], y0=r32["y"], omega0=r32["omega"])
    assert r["status"] == pdhg.STATUS_OPTIMAL
    fun = float(g["fun"][3])
    assert abs(r["metrics"]["objective"] - fun) <= 1e-6 * max(1.0, abs(fun))


def test_community_restatement_matches_highs(golden_dir):
    g = np.load(golden_dir / "highs_community.npz")
    models = syn.community_models()
    medium, biomass = syn.initial_environments(4)
    for k, mdl in enumerate(models):
        lo = dfba.uptake_lower_bounds(mdl, medium, biomass, 0.05)
        P = pdhg.prepare(mdl.S)
        r = pdhg.solve(P, lo[0], mdl.upper, mdl.cost)
        fun = float(g[f"s{k}_fun"][0])
        assert r["status"] == pdhg.STATUS_OPTIMAL
        assert abs(r["metrics"]["objective"] - fun) <= 1e-6 * max(1.0, abs(fun))


def test_uptake_bounds_follow_michaelis_menten():
    models = syn.community_models()
    mdl = models[1]
    medium = np.full((1, syn.MEDIUM_SIZE), 0.5)
    biomass = np.array([[0.05, 0.02, 0.03]])
    lo = dfba.uptake_lower_bounds(mdl, medium, biomass, 0.05)
    k = 3
    c = 0.5
    v_kin = mdl.vmax[k] * c / (mdl.km[k] + c)
    v_phys = min(c / (0.1 * 0.05), 10 * mdl.vmax[k])
    assert lo[0, mdl.medium_columns[k]] == pytest.approx(round(-min(v_kin, v_phys), 6))
    others = np.setdiff1d(np.arange(mdl.S.shape[1]), mdl.medium_columns)
    np.testing.assert_array_equal(lo[0, others], mdl.lower[others])


def test_recentred_restatement_matches_highs_and_fp64(golden_dir):
    """FP32 iterations re-centred on an FP64 base reach the FP64 tolerances in
    the same number of iterations as FP64 iterates (plain FP32 iterates stall
    near a 1e-4 gap), and the optimum matches HiGHS."""
    g = np.load(golden_dir / "highs_community.npz")
    models = syn.community_models()
    medium, biomass = syn.initial_environments(4)
    mdl = models[2]
    lo = dfba.uptake_lower_bounds(mdl, medium, biomass, 0.05)
    P = pdhg.prepare(mdl.S)
    r = pdhg.solve_recentred(P, lo[0], mdl.upper, mdl.cost)
    r64 = pdhg.solve(P, lo[0], mdl.upper, mdl.cost)
    assert r["status"] == pdhg.STATUS_OPTIMAL and r64["status"] == pdhg.STATUS_OPTIMAL
    assert abs(r["iterations"] - r64["iterations"]) <= 64
    fun = float(g["s2_fun"][0])
    assert abs(r["metrics"]["objective"] - fun) <= 1e-6 * max(1.0, abs(fun))
    cert = certificate.certificate(mdl.S, np.zeros(mdl.S.shape[0]), lo[0], mdl.upper, mdl.cost,
                                   mdl.S.shape[0], r["x"], r["y"])
    assert cert["certificate_passed"]
    plain = pdhg.solve(P, lo[0], mdl.upper, mdl.cost, dtype=np.float32, max_iters=r["iterations"] + 512,
                       stall_checks=0)
    assert plain["status"] == pdhg.STATUS_ITERATION_LIMIT


def test_recentred_handoff_finishes_in_fp64(golden_dir):
    """A re-centred solve that hands off (forced by a short stall limit)
    continues in FP64 from the handed-off point to the same optimum."""
    g = np.load(golden_dir / "highs_single.npz")
    model, lower, upper = syn.single_species_workload(8)
    P = pdhg.prepare(model.S)
    first = pdhg.solve_recentred(P, lower[1], upper[1], model.cost, handoff_stall_checks=1)
    assert first["status"] == pdhg.STATUS_HANDOFF
    r = pdhg.solve_mixed(P, lower[1], upper[1], model.cost, handoff_stall_checks=1)
    assert r["status"] == pdhg.STATUS_OPTIMAL and r["iterations"] > first["iterations"]
    fun = float(g["fun"][1])
    assert abs(r["metrics"]["objective"] - fun) <= 1e-6 * max(1.0, abs(fun))


def test_trajectory_fixture_is_pinned_to_highs_and_the_oracle(golden_dir):
    """The 48 h fixture's LP objectives agree with HiGHS at the sampled steps,
    and re-running the oracle's first steps reproduces the fixture."""
    import importlib.util
    g = np.load(golden_dir / "trajectory_community.npz")
    hs = g["highs_steps"]
    ours = g["objective"][hs]
    ref = g["highs_objective"]
    assert np.all(np.isfinite(ref))
    assert np.all(np.abs(ours - ref) <= 1e-6 * np.maximum(1.0, np.abs(ref)))
    spec = importlib.util.spec_from_file_location("make_trajectory", golden_dir / "make_trajectory.py")
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    _, states = mk.rollout(0, int(g["envs"]), 3)
    np.testing.assert_array_equal(np.array(states["objective"]), g["objective"][:3, 0])
    np.testing.assert_array_equal(states["biomass"][0][1], g["biomass"][0, 0])


def test_medium_exchange_fluxes_are_not_determined_by_the_lps():
    """Flux variability at the optimum: with the growth objective held at its
    optimum, medium exchange fluxes still span their whole bound range, so a
    metabolite trajectory depends on which optimal point a solver returns."""
    from scipy.optimize import linprog
    from scipy.sparse import csr_matrix
    models = syn.community_models()
    medium, biomass = syn.initial_environments(4, seed=11)
    mdl = models[2]
    lo = dfba.uptake_lower_bounds(mdl, medium, biomass, 0.05)[0]
    st, fun, _, _ = highs.solve_one(mdl.S, lo, mdl.upper, mdl.cost)
    kw = dict(A_eq=mdl.S, b_eq=np.zeros(mdl.S.shape[0]), A_ub=csr_matrix(mdl.cost[None, :]),
              b_ub=[fun + 1e-7 * abs(fun)], bounds=np.column_stack([lo, mdl.upper]), method="highs")
    col = int(mdl.medium_columns[0])
    e = np.zeros(mdl.S.shape[1])
    e[col] = 1.0
    vmin = linprog(e, **kw).fun
    vmax = -linprog(-e, **kw).fun
    assert vmin == pytest.approx(lo[col], abs=1e-6) and vmax == pytest.approx(mdl.upper[col], rel=1e-6)


def test_certificate_rows_equal_the_per_instance_certificate():
    """The batched certificate restates ``certificate`` row by row (equality
    and inequality rows, finite and infinite bounds)."""
    from scipy.sparse import random as sprandom
    rng = np.random.default_rng(5)
    a = sprandom(30, 50, density=0.1, random_state=6, format="csr")
    neq = 20
    E = 7
    X = rng.normal(size=(E, 50))
    Y = rng.normal(size=(E, 30))
    lower = np.where(rng.random(50) < 0.2, -np.inf, -1.0)
    upper = np.where(rng.random(50) < 0.2, np.inf, 1.0)
    c = rng.normal(size=(E, 50))
    rhs = rng.normal(size=(E, 30))
    p, d, g = certificate.certificate_rows(a, rhs, lower, upper, c, neq, X, Y)
    for i in range(E):
        ref = certificate.certificate(a, rhs[i], lower, upper, c[i], neq, X[i], Y[i])
        assert p[i] == pytest.approx(ref["primal_residual"], rel=1e-13)
        assert d[i] == pytest.approx(ref["dual_violation"], rel=1e-13)
        assert g[i] == pytest.approx(ref["relative_kkt_gap"], rel=1e-12)
