"""The parsimonious second stage of the FBA step (host side, no GPU): the
package's stage-2 LP (``parsimonious.stage_matrix`` / ``stage_bounds`` /
``stage_cost``) and the oracle's independent restatement
(``oracle.dfba.parsimonious_fluxes``) have the same optimum, which is
unique in the exchange fluxes (dual simplex and interior point agree)."""
import numpy as np
from scipy.optimize import linprog

from co_cultivation_metabolic_atlas_b200 import parsimonious as pm
from co_cultivation_metabolic_atlas_b200 import synthetic as syn
from oracle import dfba, highs


def test_stage_lp_structure():
    models = syn.community_models(sizes=((120, 300),), seed=syn.BINDING_SEED, conserved=True)
    m = models[0]
    a = pm.stage_matrix(m)
    k = m.n_exchange
    assert a.shape == (m.S.shape[0] + 2 * k, m.S.shape[1] + k)
    np.testing.assert_array_equal(a[:m.S.shape[0], :m.S.shape[1]].toarray(), m.S.toarray())
    lo, up = pm.stage_bounds(m, m.lower[None], m.upper, np.array([5.0]))
    assert lo[0, m.biomass] == max(m.lower[m.biomass], 5.0 * (1 - pm.GROWTH_RELAXATION) - pm.GROWTH_FLOOR_ABS)
    assert (lo[0, m.S.shape[1]:] == 0).all()
    np.testing.assert_array_equal(up[0, m.S.shape[1]:], np.maximum(np.abs(m.lower[:k]), np.abs(m.upper[:k])))
    w = pm.exchange_weights(m, 0)
    assert w.min() >= 1.0 and w.max() <= 10.0 and np.unique(w).size == k


def test_package_lp_equals_oracle_restatement_and_is_unique():
    models = syn.community_models(seed=syn.BINDING_SEED, conserved=True)
    medium, biomass = syn.initial_environments(2, seed=1)
    m = models[2]
    lo = dfba.uptake_lower_bounds(m, medium, biomass, 0.05)[0]
    st, fun, x, _ = highs.solve_one(m.S, lo, m.upper, m.cost)
    growth = x[m.biomass]
    status, v = dfba.parsimonious_fluxes(m, 2, lo, m.upper, growth)
    assert st == 0 and status == 0
    a = pm.stage_matrix(m)
    l2, u2 = pm.stage_bounds(m, lo[None], m.upper, np.array([growth]))
    c2 = pm.stage_cost(m, 2)
    neq = m.S.shape[0]
    kw = dict(A_eq=a[:neq], b_eq=np.zeros(neq), A_ub=a[neq:], b_ub=np.zeros(a.shape[0] - neq),
              bounds=np.column_stack([l2[0], u2[0]]))
    r_ds = linprog(c2, method="highs-ds", **kw)
    r_ipm = linprog(c2, method="highs-ipm", **kw)
    k = m.n_exchange
    w = pm.exchange_weights(m, 2)
    assert abs(r_ds.fun - float(w @ np.abs(v[:k]))) <= 1e-7 * abs(r_ds.fun)
    np.testing.assert_allclose(r_ds.x[:k], v[:k], atol=1e-6)
    np.testing.assert_allclose(r_ipm.x[:k], v[:k], atol=1e-6)
    assert v[m.biomass] == np.float64(l2[0, m.biomass]) or abs(v[m.biomass] - l2[0, m.biomass]) <= 1e-7


def test_parsimonious_trajectory_fixture_replays_its_first_step(golden_dir):
    """The committed HiGHS trajectory fixture is what its generator makes:
    environment 0's first step (stage 1 by HiGHS, the parsimonious stage 2
    by HiGHS, the oracle's Euler updates) reproduces the fixture's state at
    step 1 and the stored stage-1 growth.  Environments evolve
    independently, so one environment suffices."""
    import importlib.util
    g = np.load(golden_dir / "trajectory_parsimonious.npz")
    spec = importlib.util.spec_from_file_location("make_parsimonious_trajectory",
                                                  golden_dir / "make_parsimonious_trajectory.py")
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    models = mk._models()
    medium = g["medium"][0][:1].copy()
    biomass = g["biomass"][0][:1].copy()
    med0, bio0 = syn.initial_environments(int(g["envs"]), seed=0)
    np.testing.assert_array_equal(medium, med0[:1])
    np.testing.assert_array_equal(biomass, bio0[:1])
    out = [mk._solve((s, dfba.uptake_lower_bounds(m, medium, biomass, mk.DT)[0])) for s, m in enumerate(models)]
    growth = np.array([o[0] for o in out])
    fluxes = [o[1][None, :] for o in out]
    mu = np.stack([f[:, m.biomass] for f, m in zip(fluxes, models)], axis=1)
    b1 = dfba.update_biomass(biomass, mu, mk.DT)
    m1 = dfba.update_medium(medium, models, fluxes, biomass, mk.DT)
    np.testing.assert_allclose(growth, g["growth_stage1"][0][0], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(b1[0], g["biomass"][1][0], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(m1[0], g["medium"][1][0], rtol=1e-7, atol=1e-10)
