"""Cooperative community LP on the GPU against the HiGHS oracle of the
reference's own formulation (stage optima, certificates of the mapped-back
solutions in the reference's units)."""

import numpy as np
import pytest
import torch

from co_cultivation_metabolic_atlas_b200 import cooperative as co
from co_cultivation_metabolic_atlas_b200 import synthetic as syn
from co_cultivation_metabolic_atlas_b200.lp_trace import certificate as host_certificate
from oracle import cooperative as oc
from oracle.highs import solve_one
from tests.test_cooperative import SMALL_SIZES, crossfeeding_members, oracle_args, random_state

pytestmark = pytest.mark.gpu

# the small community seed whose three members can all grow (uptake-limited
# optima 5.3, 19.4, 3.9 at default bounds), so that the max-min growth and
# the exchanges are not trivially zero
GROWING_SMALL_SEED = 17


def reference_solution(solver, key, i, optimize, aggregate):
    """Environment i's last solution of stage ``key`` in the reference's
    variables and row layout (x_v = x_w / D, y_v = R y_w; empty metabolite
    rows and an absent performance row get no dual)."""
    st = solver.structure
    x, y, _, table, _ = solver._prev[key]
    x, y, table = x[i].double().cpu().numpy(), y[i].double().cpu().numpy(), table[i].cpu().numpy()
    stage3 = key == "parsimonious_exchange"
    rg = st.row_group3 if stage3 else st.row_group1
    cg = st.col_group3 if stage3 else st.col_group1
    xv = x / table[cg]
    yv = y * table[rg]
    full_k = st.neq + st.n_species + len(st.metabolites)
    keep1 = np.concatenate([np.arange(st.neq + st.n_species), st.neq + st.n_species + st.medium_rows])
    rows = np.arange(len(yv))
    if stage3:
        n_tail = 2 * st.n_aux
        perf_present = optimize and aggregate > 1e-9
        if optimize and not perf_present:
            rows = np.delete(rows, st.perf_row)
        ref_rows = np.concatenate([keep1, full_k + np.arange(int(perf_present) + n_tail)])
        m_ref = full_k + int(perf_present) + n_tail
    else:
        ref_rows, m_ref = keep1, full_k
    y_ref = np.zeros(m_ref)
    y_ref[ref_rows] = yv[rows]
    return xv, y_ref


def check_against_oracle(solver, members, lower, upper, biomass, medium, dt, res, *, gmax, optimize, envs):
    st, blocks, growth, exchange, orig = oracle_args(members)
    for i in envs:
        bio = dict(enumerate(biomass[i]))
        med = dict(zip(st.metabolites, medium[i]))
        full = oc.solve(blocks, growth, exchange, st.global_objective, lower[i], upper[i], bio, med, dt,
                        original_lower=orig, maximum_coexistence_growth=gmax,
                        optimize_live_objectives=optimize)
        assert full.status == "optimal"
        nu = float(res.coexistence[i])
        assert nu == pytest.approx(full.coexistence, abs=1e-6 * (1 + abs(full.coexistence)))
        agg = float(res.aggregate[i])
        probs = oc.stage_problems(blocks, growth, exchange, st.global_objective, lower[i], upper[i], bio, med, dt,
                                  coexistence=nu, aggregate=agg, original_lower=orig,
                                  maximum_coexistence_growth=gmax, optimize_live_objectives=optimize)
        keys = ["max_min"] + (["aggregate_objective"] if optimize else []) + ["parsimonious_exchange"]
        for key in keys:
            prob = probs[key]
            xv, yv = reference_solution(solver, key, i, optimize, agg)
            cert = host_certificate(prob, xv, yv)
            assert cert["certificate_passed"], (key, i, cert)
            if key != "max_min":
                status, fun, _, _ = solve_one(prob[0], prob[2], prob[3], prob[4], prob[1], prob[5])
                assert status == 0
                mine = float(prob[4] @ xv)
                assert mine == pytest.approx(fun, rel=1e-6, abs=1e-7), (key, i)


def test_crossfeeding_community_on_gpu():
    members, lower, upper = crossfeeding_members()
    solver = co.CooperativeSolver(members)
    st = solver.structure
    assert st.metabolites == ["carbon_e", "factor_e"]
    biomass = np.array([[1.0, 1.0], [1.0, 0.7], [0.23, 1.9], [0.5, 0.05]])
    medium = np.array([[10.0, 0.0], [10.0, 0.0], [2.0, 0.4], [5.0, 1.0]])
    E = len(biomass)
    lo, up = np.repeat(lower[None], E, 0), np.repeat(upper[None], E, 0)
    res = solver.solve(biomass, medium, 0.2, lo, up)
    torch.cuda.synchronize()
    assert bool(res.ok.all()), res.stages["max_min"]["status"]
    assert (res.stage.cpu() == co.STAGE_PARSIMONIOUS).all()
    v = res.fluxes.cpu().numpy()
    # without factor in the medium the consumer lives on the producer's
    # secretion in the same interval
    produced, consumed = biomass[:2, 0] * v[:2, 4], -biomass[:2, 1] * v[:2, 6]
    assert (produced > 0).all() and (consumed > 0).all() and (consumed <= produced + 1e-8).all()
    assert (v[:, 8] > 0).all()
    check_against_oracle(solver, members, lo, up, biomass, medium, 0.2, res, gmax=None, optimize=False,
                         envs=range(E))
    solver.close()


@pytest.mark.parametrize("optimize", [False, True])
def test_synthetic_community_stages_match_oracle(optimize):
    models = syn.community_models(SMALL_SIZES, seed=GROWING_SMALL_SEED, n_medium=12, per_species=6)
    members = co.synthetic_members(models)
    gmax = None if optimize else 0.005
    solver = co.CooperativeSolver(members, optimize_live_objectives=optimize, maximum_coexistence_growth=gmax)
    st = solver.structure
    rng = np.random.default_rng(11)
    E = 12
    biomass, medium = random_state(st, E, rng)
    lower = np.repeat(np.concatenate([m.lower for m in models])[None], E, 0)
    upper = np.repeat(np.concatenate([m.upper for m in models])[None], E, 0)
    # uptake-limited medium exchanges, as the dFBA step sets them
    for s, m in enumerate(models):
        cols = st.col_start[s] + m.medium_columns
        lower[:, cols] = -rng.uniform(0.0, 10.0, (E, len(cols)))
    for call in range(2):
        res = solver.solve(biomass, medium, 0.1, lower, upper)
        torch.cuda.synchronize()
        assert bool(res.ok.all()), {k: v["certified"].cpu() for k, v in res.stages.items()}
        check_against_oracle(solver, members, lower, upper, biomass, medium, 0.1, res, gmax=gmax,
                             optimize=optimize, envs=range(0, E, 3))
        # the next call warm-starts from this one, rescaled to a new biomass
        biomass = biomass * rng.uniform(0.9, 1.2, biomass.shape)
        medium = medium * rng.uniform(0.8, 1.0, medium.shape)
    solver.close()


def test_cooperative_rollout_full_size_community():
    """Three steps of the cooperative dFBA on the full-size synthetic
    community (one 6,701-column joint LP per environment and stage)."""
    models = syn.community_models(seed=syn.COOPERATIVE_SEED)
    medium, biomass = syn.initial_environments(16)
    com = co.CooperativeCommunity(models, medium, biomass, dt=0.05)
    st = com.solver.structure
    members = com.solver.structure.members
    for step in range(3):
        X = com.biomass.cpu().numpy()
        C = com.shared_medium().cpu().numpy()
        lower = com.live_bounds()
        lo = lower.cpu().numpy()
        up = com.upper.cpu().numpy()
        res = com.step()
        torch.cuda.synchronize()
        assert bool(res.ok.all())
        if step in (0, 2):
            check_against_oracle(com.solver, members, lo, up, X, C, com.dt, res, gmax=0.005, optimize=False,
                                 envs=(0, 7))
    assert torch.isfinite(com.biomass).all() and (com.biomass > 0).all()
    assert st.template1.shape[1] == st.n_fluxes + 1
    com.close()


def test_fused_certificate_equals_the_tensor_certificate():
    """The native batched certificate (``fbalp_scaled_certificate``, one
    launch) equals the tensor-op restatement on random scaled LPs of the
    stage-3 template (patched entries, free and infinite bounds, inequality
    rows); a NaN makes its instance's three values NaN."""
    models = syn.community_models(SMALL_SIZES, seed=0, n_medium=12, per_species=6)
    st = co.CommunityStructure(co.synthetic_members(models), optimize_live_objectives=True)
    dev = torch.device("cuda")
    tpl = co._Template(st.template3, st.patch3, dev)
    rng = np.random.default_rng(7)
    E, n, m = 5, st.n3, st.m3
    T = lambda a: torch.as_tensor(a, dtype=torch.float64, device=dev).contiguous()  # noqa: E731
    x = T(rng.normal(0, 3, (E, n)))
    y = T(rng.normal(0, 1, (E, m)))
    y[:, st.neq:] = -y[:, st.neq:].abs()
    y[:, st.neq + 3] = 0.5                      # a wrong-signed inequality dual
    c = T(rng.normal(0, 1, (E, n)))
    lo = T(rng.uniform(-5, 0, (E, n)))
    up = T(rng.uniform(0, 5, (E, n)))
    up[:, -st.n_aux:] = float("inf")
    lo[:, :7] = -float("inf")
    rhs = T(rng.normal(0, 1, (E, m)))
    deltas = T(rng.normal(0, 0.3, (E, len(st.patch3[0]))))
    table = T(rng.uniform(0.05, 2.0, (E, st.n_species + 3)))
    rg = torch.as_tensor(st.row_group3, device=dev)
    cg = torch.as_tensor(st.col_group3, device=dev)
    want = co.certificate(tpl, deltas, x, y, c, lo, up, rhs, st.neq, table[:, rg], table[:, cg])
    got = co.fused_certificate(tpl, deltas, x, y, c, lo, up, rhs, st.neq, rg.int(), cg.int(), table)
    for w, g in zip(want, got):
        np.testing.assert_allclose(g.cpu().numpy(), w.cpu().numpy(), rtol=1e-11, atol=1e-300)
    x[2, 11] = float("nan")
    got = co.fused_certificate(tpl, deltas, x, y, c, lo, up, rhs, st.neq, rg.int(), cg.int(), table)
    for g in got:
        v = g.cpu().numpy()
        assert np.isnan(v[2]) and np.isfinite(v[[0, 1, 3, 4]]).all()


@pytest.mark.parametrize("cap", [0.005, None])
def test_cooperative_rollout_lockstep_with_oracle(cap):
    """Twenty cooperative dFBA steps of the small community (4 environments):
    at every step the oracle solves each environment from the GPU's current
    state with HiGHS (the reference's exact-CPU stage sequence); the
    stage-1 optimum, the stage-3 optimum of the GPU fluxes and the biomass
    Euler update must agree."""
    from oracle import dfba as odfba
    models = syn.community_models(SMALL_SIZES, seed=GROWING_SMALL_SEED, n_medium=12, per_species=6)
    medium, biomass = syn.initial_environments(4, n_medium=12)
    com = co.CooperativeCommunity(models, medium, biomass, maximum_coexistence_growth=cap)
    st = com.solver.structure
    blocks, growth, exchange, obj, orig, col_start = oc.synthetic_terms(models)
    assert sorted(exchange) == st.metabolites
    upper = np.concatenate([m.upper for m in models])
    for step in range(20):
        X = com.biomass.cpu().numpy()
        C = com.medium.cpu().numpy()
        res = com.step()
        torch.cuda.synchronize()
        assert bool(res.ok.all()), step
        flux = res.fluxes.cpu().numpy()
        mu_gpu = flux[:, st.growth_cols]
        lower = np.concatenate([odfba.uptake_lower_bounds(m, C, X, com.dt) for m in models], axis=1)
        for e in range(4):
            med = {f"m{i:03d}_e": C[e, i] for i in range(C.shape[1])}
            sol = oc.solve(blocks, growth, exchange, obj, lower[e], upper, dict(enumerate(X[e])), med, com.dt,
                           original_lower=orig, maximum_coexistence_growth=cap)
            assert sol.status == "optimal"
            nu = float(res.coexistence[e])
            assert nu == pytest.approx(sol.coexistence, rel=1e-6, abs=1e-9), (step, e)
            # the GPU fluxes are optimal for the oracle's stage-3 LP
            probs = oc.stage_problems(blocks, growth, exchange, obj, lower[e], upper, dict(enumerate(X[e])), med,
                                      com.dt, coexistence=nu, original_lower=orig, maximum_coexistence_growth=cap)
            a3, b3, l3, u3, c3, neq = probs["parsimonious_exchange"]
            n = st.n_fluxes
            t = np.abs(a3[neq + st.n_species + len(st.metabolites)::2, :n] @ flux[e])
            mine = float(t.sum())
            assert mine == pytest.approx(sol.stages["parsimonious_exchange"].fun, rel=1e-6, abs=1e-7), (step, e)
        want = odfba.update_biomass(X, mu_gpu, com.dt)
        np.testing.assert_allclose(com.biomass.cpu().numpy(), want, rtol=1e-12)
    com.close()


def test_reference_style_callers_through_the_bridge():
    """The reference's exact-backend cooperative stage sequence, written as
    per-environment code calling ``backend.solve(objective, **linprog
    kwargs)`` with the reference's own assembly (oracle restatement), for
    four states of the reference's cross-feeding pair, run through
    ``BatchingBridge`` onto ``B200LPBackend``: one batched GPU solve per
    stage round, optima equal to HiGHS."""
    from scipy.sparse import block_diag, csr_matrix, hstack

    from co_cultivation_metabolic_atlas_b200 import B200LPBackend
    from co_cultivation_metabolic_atlas_b200.bridge import BatchingBridge
    members, lower, upper = crossfeeding_members()
    st, blocks, growth, exchange, orig = oracle_args(members)
    obj = st.global_objective
    biomass = np.array([[1.0, 1.0], [1.0, 0.7], [0.23, 1.9], [0.5, 0.05]])
    media = [{"carbon_e": 10.0, "factor_e": 0.0}, {"carbon_e": 10.0, "factor_e": 0.0},
             {"carbon_e": 2.0, "factor_e": 0.4}, {"carbon_e": 5.0, "factor_e": 1.0}]
    a_flux = block_diag([csr_matrix(b) for b in blocks], format="csr")
    n = a_flux.shape[1]
    a_eq = hstack([a_flux, csr_matrix((a_flux.shape[0], 1))], format="csr")
    ex_cols = [i for terms in exchange.values() for _, i, _ in terms]

    def environment(e):
        def run(backend):
            bio = dict(enumerate(biomass[e]))
            lo, up = oc.relaxed_bounds(lower, upper, ex_cols, orig, 20.0)
            a_ub, b_ub = oc.community_inequalities(n, growth, exchange, bio, media[e], 0.2)
            bounds = [(float(a), float(b)) for a, b in zip(lo, up)] + [(0.0, 10.0)]
            c1 = np.zeros(n + 1)
            c1[-1] = -1.0
            s1 = backend.solve(c1, A_ub=a_ub, b_ub=b_ub, A_eq=a_eq, b_eq=np.zeros(a_eq.shape[0]), bounds=bounds,
                               method="highs")
            assert s1.success, s1.message
            nu = max(0.0, float(s1.x[-1]))
            bounds[-1] = (nu * 0.99, nu * 0.99)
            c3, a3, b3, e3 = oc.parsimonious_lp(a_ub, b_ub, a_eq, n, exchange, bio, obj, 0.0, False, 0.99)
            s3 = backend.solve(c3, A_ub=a3, b_ub=b3, A_eq=e3, b_eq=np.zeros(e3.shape[0]),
                               bounds=bounds + [(0.0, None)] * (len(c3) - n - 1), method="highs")
            assert s3.success, s3.message
            return nu, float(s3.fun)
        return run

    parent = B200LPBackend(mode="cold", iterations=100_000, fp32_iterations=100_000)
    bridge = BatchingBridge(parent)
    res = bridge.run({e: environment(e) for e in range(4)})
    parent.close()
    assert bridge.rounds == [4, 4]
    for e, (nu, fun3) in res.items():
        sol = oc.solve(blocks, growth, exchange, obj, lower, upper, dict(enumerate(biomass[e])), media[e], 0.2,
                       original_lower=orig)
        assert nu == pytest.approx(sol.coexistence, rel=1e-6, abs=1e-9)
        assert fun3 == pytest.approx(sol.stages["parsimonious_exchange"].fun, rel=1e-5, abs=1e-7)


def test_stalled_environments_finish_in_a_second_pass():
    """In the binding regime (small community, growth cap lifted) a few of
    1,024 stage-3 LPs stop at the first pass's iteration cap; they continue
    alone from their iterates and certify, with the optima of HiGHS."""
    from oracle import dfba as odfba
    models = syn.community_models(SMALL_SIZES, seed=GROWING_SMALL_SEED, n_medium=12, per_species=6)
    medium, biomass = syn.initial_environments(1024, n_medium=12)
    com = co.CooperativeCommunity(models, medium, biomass, maximum_coexistence_growth=None)
    X = com.biomass.cpu().numpy()
    res = com.step()
    torch.cuda.synchronize()
    retried = com.solver.last_retried.get("parsimonious_exchange", [])
    assert bool(res.ok.all()), (int(res.ok.sum()), retried)
    assert retried, "no environment needed the second pass in this sample"
    st = com.solver.structure
    blocks, growth, exchange, obj, orig, _ = oc.synthetic_terms(models)
    upper = np.concatenate([m.upper for m in models])
    Cm = medium                          # the state the step started from
    lower = np.concatenate([odfba.uptake_lower_bounds(m, Cm, X, com.dt) for m in models], axis=1)
    flux = res.fluxes.cpu().numpy()
    for e in retried[:3]:
        med = {f"m{i:03d}_e": Cm[e, i] for i in range(Cm.shape[1])}
        sol = oc.solve(blocks, growth, exchange, obj, lower[e], upper, dict(enumerate(X[e])), med, com.dt,
                       original_lower=orig)
        assert sol.status == "optimal"
        probs = oc.stage_problems(blocks, growth, exchange, obj, lower[e], upper, dict(enumerate(X[e])), med, com.dt,
                                  coexistence=float(res.coexistence[e]), original_lower=orig)
        a3, _, _, _, _, neq = probs["parsimonious_exchange"]
        t = np.abs(a3[neq + st.n_species + len(st.metabolites)::2, :st.n_fluxes] @ flux[e])
        assert float(t.sum()) == pytest.approx(sol.stages["parsimonious_exchange"].fun, rel=1e-5, abs=1e-7)
    com.close()
