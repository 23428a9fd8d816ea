"""Cooperative (shared-medium) community LP restated on the CPU -- TEST
INFRASTRUCTURE ONLY (it checks the results of the batched GPU solver in
``co_cultivation_metabolic_atlas_b200.cooperative``).

Restates, in flux space ``v`` exactly as the reference assembles it,
``CooperativeCommunityFbaSolver.solve`` (``src/community_solver.py:1207-1844``)
for one environment with the exact CPU backend (HiGHS through
``scipy.optimize.linprog``):

* columns: every member's fluxes (members in order), then the coexistence
  growth ``nu`` (``:804-817``); equalities ``S_s v_s = 0`` (block diagonal);
* shared-medium inequalities ``_community_inequalities`` (``:1084-1151``):
  one growth row per member ``nu - c_s v_growth <= 0`` (growth terms in
  member order), then one row per extracellular metabolite in sorted name
  order with ``row[index] += max(1e-12, X_s) * stoich`` accumulated term by
  term and exact zeros dropped; right-hand side ``1e6`` for ``h2o_e``,
  ``h_e``, ``oh1_e`` and ``max(0, C) / dt`` otherwise;
* bounds ``_bounds`` (``:976-1022``): an exchange whose original lower bound
  is negative gets ``lower = min(lower, max(original_lower,
  -abs(max_crossfeed_uptake)))``; ``nu`` in ``[0, growth_upper]`` with
  ``growth_upper = 10`` unless ``maximum_coexistence_growth`` is given
  (``:1240-1244``);
* stage 1: ``max nu`` (``:1712-1729``); ``coexistence = max(0, nu*)``;
* stage 2 (``optimize_live_objectives``): ``nu`` in ``[floor, coexistence]``
  with ``floor = coexistence * coexistence_fraction``, maximise the live
  objectives (``:1731-1752``); otherwise ``nu`` is fixed at ``floor`` and the
  stage-1 solution is kept (``:1753-1759``);
* stage 3 (``parsimonious_exchange`` and at least one exchange variable):
  ``_assemble_parsimonious_exchange_lp`` (``:116-204``): one auxiliary
  ``t_j >= 0`` per exchange variable (dictionary order of the exchange
  terms), rows ``A_ub``, then the performance row ``-g.v <= -aggregate *
  objective_fraction`` when ``optimize_live_objectives`` and ``aggregate >
  1e-9``, then ``+-max(1e-12, X_s) stoich_j v_j - t_j <= 0``; minimise
  ``sum t`` (``:1761-1802``).

``exchange_terms`` maps a metabolite id to a list of ``(species, column,
stoich)`` in the reference's insertion order; ``growth_terms`` is a list of
``(species, column, coefficient)`` in member order.
"""

from __future__ import annotations

import operator
from dataclasses import dataclass, field

import numpy as np
from scipy.optimize import linprog
from scipy.sparse import block_diag, csr_matrix, hstack, vstack

RESERVED = frozenset({"h2o_e", "h_e", "oh1_e"})


def _column(value, n_columns):
    """NumPy scalar index semantics (negative aliases), as the dense rows of
    ``src/community_solver.py:1106-1111``."""
    value = operator.index(value)
    if value < 0:
        value += n_columns
    if value < 0 or value >= n_columns:
        raise IndexError("community reaction index outside LP columns")
    return value


def community_inequalities(n_fluxes, growth_terms, exchange_terms, biomass, medium, dt):
    """Dense-row restatement of ``_community_inequalities``: returns
    ``(A_ub csr, b_ub)`` over ``n_fluxes + 1`` columns."""
    n_columns = n_fluxes + 1
    rows, rhs = [], []
    for _, index, coefficient in growth_terms:
        row = np.zeros(n_columns)
        row[_column(index, n_columns)] = -coefficient
        row[-1] = 1.0
        rows.append(row)
        rhs.append(0.0)
    for metabolite in sorted(exchange_terms):
        row = np.zeros(n_columns)
        for species, index, stoich in exchange_terms[metabolite]:
            row[_column(index, n_columns)] += max(1e-12, float(biomass[species])) * stoich
        rows.append(row)
        rhs.append(1e6 if metabolite in RESERVED else max(0.0, float(medium.get(metabolite, 0.0))) / dt)
    if not rows:
        return csr_matrix((0, n_columns)), np.zeros(0)
    return csr_matrix(np.vstack(rows)), np.asarray(rhs, dtype=np.float64)


def relaxed_bounds(lower, upper, exchange_columns, original_lower, max_crossfeed_uptake):
    """``_bounds`` on flat arrays: ``exchange_columns`` are the global
    columns of exchange terms; ``original_lower`` maps a column to its
    original lower bound (missing: the live lower bound).  Python scalar
    ``min``/``max`` semantics, as the reference."""
    lower = np.asarray(lower, dtype=np.float64).copy()
    upper = np.asarray(upper, dtype=np.float64)
    for col in sorted(set(exchange_columns)):
        live = float(lower[col])
        orig = float(original_lower.get(col, live))
        if orig < 0.0:
            lower[col] = min(live, max(orig, -abs(max_crossfeed_uptake)))
    return lower, upper


def exchange_variables(exchange_terms):
    return [term for terms in exchange_terms.values() for term in terms]


def parsimonious_lp(a_ub, b_ub, a_eq, n_fluxes, exchange_terms, biomass, global_objective, aggregate,
                    optimize_live_objectives, objective_fraction):
    """Dense restatement of ``_assemble_parsimonious_exchange_lp``: returns
    ``(objective, A_ub, b_ub, A_eq)`` over ``n_fluxes + 1 + n_aux`` columns."""
    variables = exchange_variables(exchange_terms)
    n_aux = len(variables)
    n_columns = n_fluxes + 1 + n_aux
    a_ub = csr_matrix(a_ub).toarray()
    ub = np.zeros((a_ub.shape[0], n_columns))
    ub[:, :a_ub.shape[1]] = a_ub
    rows, rhs = [ub], [np.asarray(b_ub, dtype=np.float64)]
    if optimize_live_objectives and aggregate > 1e-9:
        perf = np.zeros((1, n_columns))
        perf[0, :n_fluxes] = -np.asarray(global_objective, dtype=np.float64)
        rows.append(perf)
        rhs.append(np.array([-aggregate * objective_fraction]))
    transfer = np.zeros((2 * n_aux, n_columns))
    for j, (species, index, stoich) in enumerate(variables):
        scale = max(1e-12, float(biomass[species])) * stoich
        transfer[2 * j, index] = scale
        transfer[2 * j + 1, index] = -scale
        transfer[2 * j:2 * j + 2, n_fluxes + 1 + j] = -1.0
    rows.append(transfer)
    rhs.append(np.zeros(2 * n_aux))
    a_eq = csr_matrix(a_eq)
    eq_ext = hstack([a_eq, csr_matrix((a_eq.shape[0], n_columns - a_eq.shape[1]))], format="csr")
    objective = np.zeros(n_columns)
    objective[n_fluxes + 1:] = 1.0
    return objective, csr_matrix(np.vstack(rows)), np.concatenate(rhs), eq_ext


@dataclass
class StageResult:
    success: bool
    fun: float = np.nan
    x: np.ndarray | None = None
    y_eq: np.ndarray | None = None
    y_ub: np.ndarray | None = None


@dataclass
class CooperativeSolution:
    status: str
    coexistence: float = np.nan
    fluxes: np.ndarray | None = None            # chosen stage's v (n_fluxes)
    nu: float = np.nan
    stage: str = ""
    stages: dict = field(default_factory=dict)  # name -> StageResult
    aggregate: float = np.nan


def _linprog(objective, a_ub, b_ub, a_eq, bounds, method):
    res = linprog(objective, A_ub=a_ub, b_ub=b_ub, A_eq=a_eq, b_eq=np.zeros(a_eq.shape[0]),
                  bounds=bounds, method=method, options=dict(presolve=True))
    if res.status != 0 or res.x is None:
        return StageResult(False)
    return StageResult(True, float(res.fun), np.asarray(res.x), np.asarray(res.eqlin.marginals),
                       np.asarray(res.ineqlin.marginals))


def solve(blocks, growth_terms, exchange_terms, objective, lower, upper, biomass, medium, dt, *,
          original_lower=None, max_crossfeed_uptake=20.0, coexistence_fraction=0.99, objective_fraction=0.99,
          maximum_coexistence_growth=None, optimize_live_objectives=False, parsimonious_exchange=True,
          method="highs"):
    """One environment's cooperative solve (the exact-CPU path of
    ``src/community_solver.py:1207-1811``).  ``objective`` is the global
    objective vector (maximisation sense, ``_objective_vector``)."""
    a_flux = block_diag([csr_matrix(b) for b in blocks], format="csr")
    n_fluxes = a_flux.shape[1]
    a_eq = hstack([a_flux, csr_matrix((a_flux.shape[0], 1))], format="csr")
    ex_cols = [index for terms in exchange_terms.values() for _, index, _ in terms]
    lo, up = relaxed_bounds(lower, upper, ex_cols, original_lower or {}, max_crossfeed_uptake)
    a_ub, b_ub = community_inequalities(n_fluxes, growth_terms, exchange_terms, biomass, medium, dt)
    gmax = 10.0 if maximum_coexistence_growth is None else max(0.0, float(maximum_coexistence_growth))
    bounds = [(float(a), float(b)) for a, b in zip(lo, up)] + [(0.0, gmax)]
    out = CooperativeSolution(status="")
    c1 = np.zeros(n_fluxes + 1)
    c1[-1] = -1.0
    s1 = _linprog(c1, a_ub, b_ub, a_eq, bounds, method)
    out.stages["max_min"] = s1
    if not s1.success:
        out.status = "coexistence_infeasible"
        return out
    coexistence = max(0.0, float(s1.x[-1]))
    out.coexistence = coexistence
    floor = coexistence * float(np.clip(coexistence_fraction, 0.0, 1.0))
    bounds2 = list(bounds)
    g = np.asarray(objective, dtype=np.float64)
    if optimize_live_objectives:
        bounds2[-1] = (floor, coexistence)
        s2 = _linprog(np.concatenate([-g, [0.0]]), a_ub, b_ub, a_eq, bounds2, method)
        out.stages["aggregate_objective"] = s2
        if not s2.success:
            out.status = "stage2_failed"
            return out
        chosen, stage = s2, "aggregate_objective"
    else:
        bounds2[-1] = (floor, floor)
        chosen, stage = s1, "max_min"
    aggregate = float(g @ chosen.x[:n_fluxes])
    out.aggregate = aggregate
    n_aux = len(exchange_variables(exchange_terms))
    if n_aux and parsimonious_exchange:
        c3, a3, b3, e3 = parsimonious_lp(a_ub, b_ub, a_eq, n_fluxes, exchange_terms, biomass, g, aggregate,
                                          optimize_live_objectives, float(np.clip(objective_fraction, 0, 1)))
        s3 = _linprog(c3, a3, b3, e3, bounds2 + [(0.0, None)] * n_aux, method)
        out.stages["parsimonious_exchange"] = s3
        if not s3.success:
            out.status = "stage3_failed"
            return out
        chosen, stage = s3, "parsimonious_exchange"
    out.status = "optimal"
    out.stage = stage
    out.fluxes = chosen.x[:n_fluxes]
    out.nu = float(chosen.x[n_fluxes])
    return out


def stage_problems(blocks, growth_terms, exchange_terms, objective, lower, upper, biomass, medium, dt, *,
                   coexistence, aggregate=0.0, original_lower=None, max_crossfeed_uptake=20.0,
                   coexistence_fraction=0.99, objective_fraction=0.99, maximum_coexistence_growth=None,
                   optimize_live_objectives=False):
    """The stage LPs of one environment as ``(A, rhs, lower, upper, c,
    neq)`` tuples (equalities first, the certificate's layout), for a given
    stage-1 optimum ``coexistence`` and stage-3 ``aggregate``."""
    a_flux = block_diag([csr_matrix(b) for b in blocks], format="csr")
    n_fluxes = a_flux.shape[1]
    neq = a_flux.shape[0]
    a_eq = hstack([a_flux, csr_matrix((neq, 1))], format="csr")
    ex_cols = [index for terms in exchange_terms.values() for _, index, _ in terms]
    lo, up = relaxed_bounds(lower, upper, ex_cols, original_lower or {}, max_crossfeed_uptake)
    a_ub, b_ub = community_inequalities(n_fluxes, growth_terms, exchange_terms, biomass, medium, dt)
    gmax = 10.0 if maximum_coexistence_growth is None else max(0.0, float(maximum_coexistence_growth))
    g = np.asarray(objective, dtype=np.float64)
    floor = coexistence * float(np.clip(coexistence_fraction, 0.0, 1.0))
    out = {}
    c1 = np.zeros(n_fluxes + 1)
    c1[-1] = -1.0
    lo1, up1 = np.append(lo, 0.0), np.append(up, gmax)
    out["max_min"] = (vstack([a_eq, a_ub], format="csr"), np.concatenate([np.zeros(neq), b_ub]), lo1, up1, c1, neq)
    nu_hi = coexistence if optimize_live_objectives else floor
    lo2, up2 = np.append(lo, floor), np.append(up, nu_hi)
    if optimize_live_objectives:
        out["aggregate_objective"] = (out["max_min"][0], out["max_min"][1], lo2, up2,
                                      np.concatenate([-g, [0.0]]), neq)
    c3, a3, b3, e3 = parsimonious_lp(a_ub, b_ub, a_eq, n_fluxes, exchange_terms, biomass, g, aggregate,
                                      optimize_live_objectives, float(np.clip(objective_fraction, 0, 1)))
    n_aux = len(c3) - n_fluxes - 1
    out["parsimonious_exchange"] = (vstack([e3, a3], format="csr"), np.concatenate([np.zeros(neq), b3]),
                                    np.concatenate([lo2, np.zeros(n_aux)]),
                                    np.concatenate([up2, np.full(n_aux, np.inf)]), c3, neq)
    return out


def synthetic_terms(models, secondary=60, seed=0):
    """The cooperative LP data of the synthetic community, restated: every
    exchange column is an exchange term (stoichiometry -1) -- a medium column
    of its medium metabolite ``m{id:03d}_e``, every other exchange column of
    one of ``secondary`` shared metabolites ``m{100+k:03d}_e`` (seeded
    draws, generator ``default_rng(seed + 4242)``, in species then column
    order), absent from the medium; original bounds = the default lower
    bounds; the growth reaction is the biomass column (coefficient 1); the
    objective maximises biomass.  Returns ``(blocks, growth_terms,
    exchange_terms, objective, original_lower, col_start)``."""
    rng = np.random.default_rng(seed + 4242)
    col_start = np.concatenate([[0], np.cumsum([m.S.shape[1] for m in models])]).astype(int)
    growth, exchange, orig, obj = [], {}, {}, []
    for s, m in enumerate(models):
        growth.append((s, int(col_start[s] + m.biomass), 1.0))
        medium = {int(c): int(i) for c, i in zip(m.medium_columns, m.medium_ids)}
        others = [c for c in range(m.n_exchange) if c not in medium]
        draw = rng.integers(0, secondary, len(others))
        ids = dict(medium)
        for c, k in zip(others, draw):
            ids[c] = 100 + int(k)
        for c in range(m.n_exchange):
            gcol = int(col_start[s] + c)
            exchange.setdefault(f"m{ids[c]:03d}_e", []).append((s, gcol, -1.0))
            if m.lower[c] < 0:
                orig[gcol] = float(m.lower[c])
        obj.append(-np.asarray(m.cost, dtype=float))
    return [m.S for m in models], growth, exchange, np.concatenate(obj), orig, col_start
