"""Cooperative community LP: oracle pins against the reference's own tests
and exactness of the biomass-scaled formulation (CPU only)."""

import numpy as np
import pytest
import torch
from scipy.sparse import csr_matrix

from co_cultivation_metabolic_atlas_b200 import cooperative as co
from co_cultivation_metabolic_atlas_b200 import synthetic as syn
from co_cultivation_metabolic_atlas_b200.lp_trace import certificate as host_certificate
from oracle import cooperative as oc

SMALL_SIZES = ((80, 260), (90, 280), (70, 240))


# -- oracle pins ---------------------------------------------------------------

def test_inequality_assembly_pin():
    """Known answer of ``tests/test_community_inequality_assembly.py``: its
    growth/exchange fixture at biomass a=1, b=0.7, medium glucose 0.3, z -4,
    dt 0.2 (rows: growth b, growth a, then sorted metabolites; the
    (1e16 - 1e16) + 1 sum stays 1; the cancelling row is empty)."""
    growth = [("b", 3, 0.75), ("a", 0, 1.0)]
    exchange = {
        "z": [("a", 2, 1e16), ("b", 4, -0.25), ("a", 2, -1e16), ("a", 2, 1.0)],
        "h_e": [("a", 1, -1.0)],
        "empty": [],
        "glucose": [("a", 0, -0.1), ("b", 3, -0.3)],
        "cancels": [("a", 1, 0.5), ("a", 1, -0.5), ("b", 4, 0.0)],
        "h2o_e": [("a", 2, -1.0)],
        "oh1_e": [("b", 4, -1.0)],
    }
    a, b = oc.community_inequalities(5, growth, exchange, {"a": 1.0, "b": 0.7},
                                     {"glucose": 0.3, "z": -4.0, "h_e": 0.0}, 0.2)
    want = np.zeros((9, 6))
    want[0, 3], want[0, 5] = -0.75, 1.0
    want[1, 0], want[1, 5] = -1.0, 1.0
    # sorted: cancels, empty, glucose, h2o_e, h_e, oh1_e, z
    want[4, 0], want[4, 3] = -0.1, 0.7 * -0.3
    want[5, 2] = -1.0
    want[6, 1] = -1.0
    want[7, 4] = -0.7
    want[8, 2], want[8, 4] = 1.0, 0.7 * -0.25
    np.testing.assert_array_equal(a.toarray(), want)
    np.testing.assert_array_equal(b, [0, 0, 0, 0, 0.3 / 0.2, 1e6, 1e6, 1e6, 0])
    assert a[2].nnz == 0 and a[3].nnz == 0
    # the biomass floor: a member at zero biomass contributes 1e-12 * stoich
    a0, _ = oc.community_inequalities(5, growth, exchange, {"a": 0.0, "b": -3.0}, {}, 0.2)
    assert a0[4, 0] == pytest.approx(-0.1e-12) and a0[4, 3] == pytest.approx(-0.3e-12)


@pytest.mark.parametrize("maximum", [0.0, 0.1, 4.0, -4.0, np.inf, np.nan])
def test_crossfeed_relaxation_pin(maximum):
    """The live-bound rule of ``tests/test_community_bounds_packing.py``:
    exchanges whose ORIGINAL lower bound is negative are widened to
    ``max(original, -|limit|)``; others keep their live bounds."""
    lower = np.array([-0.1, -np.inf, 0.0, 0.0, -3.0, -0.2])
    upper = np.array([1000.0, np.inf, 0.0, 2.0, 7.0, 4.0])
    lo, up = oc.relaxed_bounds(lower, upper, [0, 2, 5], {0: -8.0, 2: 0.0, 5: -3.0}, maximum)
    cap0 = max(-8.0, -abs(maximum))
    cap5 = max(-3.0, -abs(maximum))
    assert lo[0] == min(-0.1, cap0) and lo[5] == min(-0.2, cap5)
    np.testing.assert_array_equal(lo[[1, 2, 3, 4]], lower[[1, 2, 3, 4]])
    np.testing.assert_array_equal(up, upper)


def crossfeeding_members():
    """The producer / consumer pair of ``tests/test_community_solver.py``
    (``_crossfeeding_models``): the producer turns carbon into a secreted
    factor, the consumer grows only on that factor."""
    # producer: rows carbon_e, carbon_c, factor_c, factor_e;
    # columns EX_carbon, carbon_transport, make_factor, factor_export, EX_factor, Growth
    p = np.zeros((4, 6))
    p[0, 0] = -1
    p[0, 1], p[1, 1] = -1, 1
    p[1, 2], p[2, 2] = -2, 1
    p[2, 3], p[3, 3] = -1, 1
    p[3, 4] = -1
    p[1, 5] = -1
    # consumer: rows factor_e, factor_c; columns EX_factor, factor_import, Growth
    c = np.zeros((2, 3))
    c[0, 0] = -1
    c[0, 1], c[1, 1] = -1, 1
    c[1, 2] = -1
    producer = co.Member("producer", csr_matrix(p), growth=5, objective=np.eye(6)[5],
                         exchanges=(("carbon_e", 0, -1.0), ("factor_e", 4, -1.0)),
                         original_lower={0: -10.0, 4: 0.0})
    consumer = co.Member("consumer", csr_matrix(c), growth=2, objective=np.eye(3)[2],
                         exchanges=(("factor_e", 0, -1.0),), original_lower={0: -10.0})
    lower = np.array([-10, 0, 0, 0, 0, 0, 0, 0, 0], float)     # the consumer's own EX_factor closed
    upper = np.array([1000, 1000, 1000, 1000, 1000, 1000, 1000, 1000, 1000], float)
    return [producer, consumer], lower, upper


def oracle_args(members):
    st = co.CommunityStructure(members)
    growth = [(s, int(st.growth_cols[s]), float(st.growth_coef[s])) for s in range(st.n_species)]
    exchange = {met: [(s, c, v) for s, c, v in terms] for met, terms in st.exchange_terms.items()}
    orig = {int(c): o for c, o in zip(st.relax_cols, st.relax_orig)}
    return st, [m.S for m in members], growth, exchange, orig


def test_crossfeeding_oracle_matches_reference_test():
    """``test_cooperative_solver_enables_mass_balanced_same_step_crossfeeding``:
    with the shared pool the consumer grows on the producer's factor."""
    members, lower, upper = crossfeeding_members()
    st, blocks, growth, exchange, orig = oracle_args(members)
    sol = oc.solve(blocks, growth, exchange, st.global_objective, lower, upper, {0: 1.0, 1: 1.0},
                   {"carbon_e": 10.0, "factor_e": 0.0}, 1.0, original_lower=orig)
    assert sol.status == "optimal"
    v = sol.fluxes
    produced, consumed = v[4], -v[6]
    assert produced > 0.0 and consumed > 0.0
    assert consumed <= produced + 1e-8
    assert v[8] > 0.0


# -- the scaled formulation ------------------------------------------------------

def synthetic_small(seed=0):
    models = syn.community_models(SMALL_SIZES, seed=seed, n_medium=12, per_species=6)
    return co.synthetic_members(models), models


def random_state(st, E, rng):
    biomass = rng.uniform(0.01, 2.0, (E, st.n_species))
    medium = rng.lognormal(0.0, 1.0, (E, len(st.metabolites)))
    return biomass, medium


def patched_matrix(template, patch, deltas_row):
    a = template.tolil(copy=True)
    for r, c, d in zip(patch[0], patch[1], deltas_row):
        a[r, c] = a[r, c] + d
    return a.tocsr()


@pytest.mark.parametrize("optimize", [False, True])
@pytest.mark.parametrize("which", ["crossfeeding", "synthetic"])
def test_scaled_lp_is_the_reference_lp_under_diagonal_scalings(which, optimize):
    """For every environment, the engine's LP (shared template + patched
    deltas) equals R A_ref D^-1 with b = R b_ref, bounds D l_ref, cost
    D^-1 c_ref, where A_ref etc. are assembled exactly as the reference
    does (stage 1 and stage 3)."""
    rng = np.random.default_rng(3)
    if which == "crossfeeding":
        members, lower, upper = crossfeeding_members()
    else:
        members, models = synthetic_small()
        lower = np.concatenate([m.lower for m in models])
        upper = np.concatenate([m.upper for m in models])
    st = co.CommunityStructure(members, optimize_live_objectives=optimize)
    _, blocks, growth, exchange, orig = oracle_args(members)
    asm = co.StageAssembly(st, "cpu")
    E = 3
    biomass, medium = random_state(st, E, rng)
    dt = 0.2
    T = lambda a: torch.as_tensor(a, dtype=torch.float64)  # noqa: E731
    lo = asm.relaxed_lower(T(np.repeat(lower[None], E, 0)), 20.0)
    sc = asm.scales(T(biomass))
    lw, uw, l1, u1, c1, rhs1, d1 = asm.stage1(sc, lo, T(np.repeat(upper[None], E, 0)), T(medium), dt, 0.005)
    coexistence = torch.full((E,), 0.004, dtype=torch.float64)
    floor = coexistence * 0.99
    l2, u2, c2 = asm.stage2(sc, lw, uw, floor, coexistence if optimize else floor)
    aggregate = T(rng.uniform(0.0, 2.0, E))
    aggregate[0] = 0.0                        # the performance row is absent
    l3, u3, c3, rhs3, d3 = asm.stage3(sc, l2, u2, rhs1, d1, aggregate, 0.99)
    keep1 = np.concatenate([np.arange(st.neq + st.n_species), st.neq + st.n_species + st.medium_rows])
    for i in range(E):
        probs = oc.stage_problems(blocks, growth, exchange, st.global_objective, lower, upper,
                                  dict(enumerate(biomass[i])), dict(zip(st.metabolites, medium[i])), dt,
                                  coexistence=float(coexistence[i]), aggregate=float(aggregate[i]),
                                  original_lower=orig, maximum_coexistence_growth=0.005,
                                  optimize_live_objectives=optimize)
        cases = [("max_min", st.template1, st.patch1, d1, (l1, u1, c1, rhs1), keep1, st.row_group1, st.col_group1)]
        if optimize:
            cases.append(("aggregate_objective", st.template1, st.patch1, d1, (l2, u2, c2, rhs1), keep1,
                          st.row_group1, st.col_group1))
        cases.append(("parsimonious_exchange", st.template3, st.patch3, d3, (l3, u3, c3, rhs3), None,
                      st.row_group3, st.col_group3))
        full_k = st.neq + st.n_species + len(st.metabolites)
        for name, tpl, patch, deltas, (lw_, uw_, cw_, bw_), keep, rg, cg in cases:
            a_ref, b_ref, l_ref, u_ref, c_ref, neq = probs[name]
            a_w = patched_matrix(tpl, patch, deltas[i].numpy()).toarray()
            R = sc.table[i, torch.as_tensor(rg)].numpy()
            D = sc.table[i, torch.as_tensor(cg)].numpy()
            bw = bw_[i].numpy()
            a_ref = a_ref.toarray()
            if keep is not None:
                ref_rows = keep
            else:
                # the reference's rows after all its metabolite rows: the
                # performance row (when present) and the transfer rows
                ref_rows = np.concatenate([keep1, np.arange(full_k, a_ref.shape[0])])
                if optimize and float(aggregate[i]) <= 1e-9:
                    # reference: no performance row; here the same row with
                    # zero coefficients and right-hand side
                    assert np.all(a_w[st.perf_row] == 0) and bw[st.perf_row] == 0
                    rows = np.delete(np.arange(st.m3), st.perf_row)
                    a_w, R, bw = a_w[rows], R[rows], bw[rows]
            a_ref, b_ref = a_ref[ref_rows], b_ref[ref_rows]
            np.testing.assert_allclose(a_w, R[:, None] * a_ref / D[None, :], rtol=1e-14, atol=1e-300)
            np.testing.assert_allclose(bw, R * b_ref, rtol=1e-14)
            np.testing.assert_allclose(lw_[i].numpy(), D * l_ref, rtol=1e-14)
            np.testing.assert_allclose(uw_[i].numpy(), D * u_ref, rtol=1e-14)
            np.testing.assert_allclose(cw_[i].numpy(), c_ref / D, rtol=1e-14)
            assert neq == st.neq


def test_certificate_of_mapped_highs_solution():
    """The scaled-LP certificate of a HiGHS solution of the reference LP,
    mapped into the scaled variables, reproduces the reference-units
    certificate of that solution."""
    members, models = synthetic_small(1)
    st = co.CommunityStructure(members)
    _, blocks, growth, exchange, orig = oracle_args(members)
    asm = co.StageAssembly(st, "cpu")
    lower = np.concatenate([m.lower for m in models])
    upper = np.concatenate([m.upper for m in models])
    rng = np.random.default_rng(5)
    E = 2
    biomass, medium = random_state(st, E, rng)
    T = lambda a: torch.as_tensor(a, dtype=torch.float64)  # noqa: E731
    sc = asm.scales(T(biomass))
    lo = asm.relaxed_lower(T(np.repeat(lower[None], E, 0)), 20.0)
    lw, uw, l1, u1, c1, rhs1, d1 = asm.stage1(sc, lo, T(np.repeat(upper[None], E, 0)), T(medium), 0.1, 10.0)
    tpl = co._Template(st.template1, st.patch1, "cpu")
    keep = np.concatenate([np.arange(st.neq + st.n_species), st.neq + st.n_species + st.medium_rows])
    xs, ys, want = [], [], []
    for i in range(E):
        a, b, l, u, c, neq = oc.stage_problems(blocks, growth, exchange, st.global_objective, lower, upper,
                                               dict(enumerate(biomass[i])), dict(zip(st.metabolites, medium[i])),
                                               0.1, coexistence=0.0, original_lower=orig)["max_min"]
        from oracle.highs import solve_one
        status, fun, x, y = solve_one(a, l, u, c, b, neq)
        assert status == 0
        want.append(host_certificate((a, b, l, u, c, neq), x, y))
        R = sc.table[i, torch.as_tensor(st.row_group1)].numpy()
        D = sc.table[i, torch.as_tensor(st.col_group1)].numpy()
        xs.append(D * x)
        ys.append(y[keep] / R)
    primal, dual, gap = co.certificate(tpl, d1, T(np.array(xs)), T(np.array(ys)), c1, l1, u1, rhs1, st.neq,
                                       sc.table[:, torch.as_tensor(st.row_group1)],
                                       sc.table[:, torch.as_tensor(st.col_group1)])
    for i in range(E):
        assert primal[i] == pytest.approx(want[i]["primal_residual"], abs=1e-9)
        assert dual[i] == pytest.approx(want[i]["dual_violation"], abs=1e-12)
        assert gap[i] == pytest.approx(want[i]["relative_kkt_gap"], abs=1e-9)
        assert primal[i] <= co.PRIMAL_GATE and dual[i] <= co.DUAL_GATE and gap[i] <= co.GAP_GATE


def test_structure_limits_and_layout():
    members, _ = synthetic_small()
    st = co.CommunityStructure(members, optimize_live_objectives=True)
    assert st.template1.shape == (st.neq + 3 + st.n_medium_rows, st.n_fluxes + 1)
    assert st.template3.shape == (st.m1 + 1 + 2 * st.n_aux, st.n_fluxes + 1 + st.n_aux)
    assert len(st.patch3[0]) == 6 <= co.N.MAX_PATCHES
    assert st.metabolites == sorted(st.metabolites)
    with pytest.raises(ValueError):
        co.CommunityStructure([co.Member("x", members[0].S, growth=10 ** 6, objective=members[0].objective)])
