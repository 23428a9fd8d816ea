"""Batched cooperative (shared-medium) community LP on the GPU.

The reference's cooperative dFBA mode solves, for every environment and
every step, up to three LPs over all members at once
(``CooperativeCommunityFbaSolver.solve``, ``src/community_solver.py:
1207-1811``):

1. max-min growth: ``max nu`` s.t. ``S_s v_s = 0``, ``nu - c_s v_growth(s)
   <= 0`` for every member, and one shared-medium row per extracellular
   metabolite ``sum_s X_s stoich v_exchange <= C / dt`` (``:1084-1151``);
2. optionally the live objectives with ``nu`` in ``[floor, coexistence]``;
3. parsimonious exchange: ``min sum t_j`` with ``t_j >= |X_s stoich_j v_j|``
   for every exchange variable (``_assemble_parsimonious_exchange_lp``,
   ``:116-204``).

The biomass ``X_s`` multiplies matrix coefficients, so every environment's
LP has its own matrix.  This module solves them with the species-shared
engine by a change of variables that moves the biomass out of the matrix:
with ``Xbar = max_s X_s`` (``X_s`` floored at 1e-12 as the reference does)
and ``rho_s = X_s / Xbar``,

    w_s = rho_s v_s,   t'_j = t_j / Xbar

turns the LP into

    S_s w_s = 0                                     (rows scaled by rho_s)
    rho_s nu - c_s w_growth(s) <= 0                 (rows scaled by rho_s)
    sum stoich w_exchange <= (C / dt) / Xbar        (rows scaled by 1 / Xbar)
    +-stoich_j w_j - t'_j <= 0                      (rows scaled by 1 / Xbar)
    -sum_j g_j (rho_min / rho_s) w_j <= -aggregate fraction rho_min
                                                    (row scaled by rho_min)
    rho_s l <= w_s <= rho_s u,   cost c_w = c_v / rho  (t': cost Xbar)

Only the ``nu`` coefficient of each growth row (and, with live objectives,
the coefficients of the performance row) depends on the environment; they
are the engine's per-instance patched entries.  Every other coefficient is
shared by all environments.  The transformed LP is the reference's LP under
positive diagonal row and column scalings: objective values, optimal faces
and complementarity are unchanged, and the solution maps back exactly.  The
certificate is evaluated in the reference's units (residuals divided by the
row scaling, reduced costs multiplied by the column scaling) with the
reference's gate.
"""

from __future__ import annotations

import ctypes
import warnings
from dataclasses import dataclass, field

import numpy as np
import torch
from scipy.sparse import block_diag, csr_matrix, hstack, vstack

from . import _native as N
from .dfba import CARRYING_CAPACITY, euler_biomass, uptake_lower
from .engine import EngineOptions, LPEngine, SolveConfig, SolveResult

RESERVED_METABOLITES = frozenset({"h2o_e", "h_e", "oh1_e"})   # src/community_solver.py:1148
RESERVED_SUPPLY = 1e6
BIOMASS_FLOOR = 1e-12
DEFAULT_GROWTH_UPPER = 10.0
PRIMAL_GATE, DUAL_GATE, GAP_GATE = 1e-5, 1e-7, 1e-7                # src/gpu_block_lp.py:84

STAGE_FAILED, STAGE_MAX_MIN, STAGE_AGGREGATE, STAGE_PARSIMONIOUS = 0, 1, 2, 3
STAGE_NAMES = {STAGE_FAILED: "failed", STAGE_MAX_MIN: "max_min", STAGE_AGGREGATE: "aggregate_objective",
               STAGE_PARSIMONIOUS: "parsimonious_exchange"}


@dataclass
class Member:
    """One community member: stoichiometry, growth reaction, live objective
    (coefficients and direction, ``_objective_vector`` ``:954-974``),
    extracellular exchange terms ``(metabolite, local column, stoich)`` and
    the original lower bounds of its exchanges (local column -> bound) for
    the cross-feeding relaxation (``_bounds`` ``:976-1022``)."""

    name: str
    S: csr_matrix
    growth: int
    objective: np.ndarray
    direction: str = "max"
    growth_coefficient: float = 1.0
    exchanges: tuple = ()
    original_lower: dict = field(default_factory=dict)

    @property
    def n(self):
        return self.S.shape[1]


class CommunityStructure:
    """Host-side structure of the transformed cooperative LPs: column and
    row layout, the shared template matrices and the patched entries."""

    def __init__(self, members, *, optimize_live_objectives=False):
        members = list(members)
        if not members:
            raise ValueError("at least one member is required")
        self.members = members
        self.optimize_live_objectives = bool(optimize_live_objectives)
        S = len(members)
        self.n_species = S
        sizes = [m.n for m in members]
        self.col_start = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        self.n_fluxes = int(self.col_start[-1])
        self.nu = self.n_fluxes
        self.col_species = np.repeat(np.arange(S), sizes)
        rows = [m.S.shape[0] for m in members]
        self.row_start = np.concatenate([[0], np.cumsum(rows)]).astype(np.int64)
        self.neq = int(self.row_start[-1])
        for m in members:
            if m.direction not in ("max", "min"):
                raise ValueError("objective direction must be 'max' or 'min'")
            if not 0 <= m.growth < m.n:
                raise ValueError(f"growth column of {m.name} out of range")
            if np.asarray(m.objective).shape != (m.n,):
                raise ValueError(f"objective of {m.name} does not match its columns")
        self.growth_cols = np.array([self.col_start[s] + m.growth for s, m in enumerate(members)], np.int64)
        self.growth_coef = np.array([float(m.growth_coefficient) for m in members])
        # per-species objective coefficients (reported objective values) and
        # the global objective in maximisation sense
        self.objectives = [np.asarray(m.objective, dtype=np.float64).copy() for m in members]
        self.global_objective = np.concatenate(
            [(-o if m.direction == "min" else o) for o, m in zip(self.objectives, members)])
        # exchange terms in the reference's insertion order (member order,
        # then each member's exchange order; ``:775-790``)
        terms: dict[str, list] = {}
        relax_cols, relax_orig = [], []
        for s, m in enumerate(members):
            for met, col, stoich in m.exchanges:
                if not 0 <= int(col) < m.n:
                    raise ValueError(f"exchange column of {m.name} out of range")
                gcol = int(self.col_start[s] + int(col))
                terms.setdefault(str(met), []).append((s, gcol, float(stoich)))
            for col, orig in m.original_lower.items():
                if any(int(c) == int(col) for _, c, _ in m.exchanges) and float(orig) < 0.0:
                    relax_cols.append(int(self.col_start[s] + int(col)))
                    relax_orig.append(float(orig))
        self.exchange_terms = terms
        self.metabolites = sorted(terms)
        self.variables = [t for met in terms for t in terms[met]]
        self.relax_cols = np.asarray(relax_cols, dtype=np.int64)
        self.relax_orig = np.asarray(relax_orig, dtype=np.float64)
        # shared-medium rows in sorted metabolite order; the coefficient of a
        # column is its accumulated stoichiometry (every column belongs to one
        # member, so the biomass factors out), exact zeros dropped; rows with
        # no coefficient left are not constraints and are not built
        med = []
        for k, met in enumerate(self.metabolites):
            acc: dict[int, float] = {}
            for _, col, stoich in terms[met]:
                acc[col] = acc.get(col, 0.0) + stoich
            entries = {c: v for c, v in acc.items() if v != 0.0}
            if entries:
                med.append((k, entries))
        self.medium_rows = np.array([k for k, _ in med], dtype=np.int64)
        self.medium_reserved = np.array([self.metabolites[k] in RESERVED_METABOLITES for k, _ in med], bool)
        K = len(med)
        self.n_medium_rows = K
        n1 = self.n_fluxes + 1
        a_eq = block_diag([csr_matrix(m.S, dtype=np.float64) for m in members], format="csr")
        eq = hstack([a_eq, csr_matrix((self.neq, 1))], format="csr")
        gr_r, gr_c, gr_v = [], [], []
        for s in range(S):
            gr_r += [s, s]
            gr_c += [int(self.growth_cols[s]), self.nu]
            gr_v += [-self.growth_coef[s], 1.0]
        growth = csr_matrix((gr_v, (gr_r, gr_c)), shape=(S, n1))
        md_r, md_c, md_v = [], [], []
        for r, (_, entries) in enumerate(med):
            for c, v in sorted(entries.items()):
                md_r.append(r)
                md_c.append(c)
                md_v.append(v)
        medium = csr_matrix((md_v, (md_r, md_c)), shape=(K, n1))
        self.template1 = vstack([eq, growth, medium], format="csr")
        self.m1 = self.template1.shape[0]
        self.n1 = n1
        self.growth_rows = self.neq + np.arange(S)
        self.patch1 = (self.growth_rows.copy(), np.full(S, self.nu, np.int64))
        # stage 3
        n_aux = len(self.variables)
        self.n_aux = n_aux
        n3 = n1 + n_aux
        self.n3 = n3
        ext = hstack([self.template1, csr_matrix((self.m1, n_aux))], format="csr")
        blocks = [ext]
        perf_cols = np.flatnonzero(self.global_objective)
        self.perf_cols = perf_cols
        self.perf_row = -1
        if self.optimize_live_objectives:
            self.perf_row = self.m1
            blocks.append(csr_matrix((-self.global_objective[perf_cols], (np.zeros(len(perf_cols), int), perf_cols)),
                                     shape=(1, n3)))
        tr_r, tr_c, tr_v = [], [], []
        for j, (_, col, stoich) in enumerate(self.variables):
            for sgn, r in ((1.0, 2 * j), (-1.0, 2 * j + 1)):
                if stoich != 0.0:
                    tr_r.append(r)
                    tr_c.append(col)
                    tr_v.append(sgn * stoich)
                tr_r.append(r)
                tr_c.append(n1 + j)
                tr_v.append(-1.0)
        blocks.append(csr_matrix((tr_v, (tr_r, tr_c)), shape=(2 * n_aux, n3)))
        self.template3 = vstack(blocks, format="csr")
        self.m3 = self.template3.shape[0]
        self.transfer_start = self.m1 + (1 if self.optimize_live_objectives else 0)
        p3r, p3c = list(self.patch1[0]), list(self.patch1[1])
        if self.optimize_live_objectives:
            p3r += [self.perf_row] * len(perf_cols)
            p3c += list(perf_cols)
        self.patch3 = (np.asarray(p3r, np.int64), np.asarray(p3c, np.int64))
        # scaling groups: a row / column is scaled by rho_s (group s), by
        # 1 / Xbar (group S), by rho_min (group S + 1) or not (group S + 2)
        self.row_group1 = np.concatenate([np.repeat(np.arange(S), rows), np.arange(S), np.full(K, S)])
        self.row_group3 = np.concatenate([self.row_group1, [S + 1] if self.optimize_live_objectives else [],
                                          np.full(2 * n_aux, S)]).astype(np.int64)
        self.col_group1 = np.concatenate([self.col_species, [S + 2]]).astype(np.int64)
        self.col_group3 = np.concatenate([self.col_group1, np.full(n_aux, S)]).astype(np.int64)
        self.var_cols = np.array([c for _, c, _ in self.variables], np.int64)
        self.var_stoich = np.array([v for _, _, v in self.variables], np.float64)


def _csr_tensor(a, device):
    a = csr_matrix(a)
    a.sort_indices()
    with warnings.catch_warnings():
        # torch flags its CSR layout as beta; the arrays come from a
        # canonical SciPy matrix
        warnings.simplefilter("ignore", UserWarning)
        return torch.sparse_csr_tensor(torch.as_tensor(a.indptr, dtype=torch.int64),
                                       torch.as_tensor(a.indices, dtype=torch.int64),
                                       torch.as_tensor(a.data, dtype=torch.float64), size=a.shape, device=device,
                                       check_invariants=False)


class _Template:
    """Device copy of a template and its transpose for the certificate."""

    def __init__(self, a, patch, device):
        self.A = _csr_tensor(a, device)
        self.AT = _csr_tensor(csr_matrix(a).T.tocsr(), device)
        self.prow = torch.as_tensor(patch[0], device=device)
        self.pcol = torch.as_tensor(patch[1], device=device)
        self.m, self.n = a.shape
        # int32 CSR arrays for the fused certificate kernel
        i32 = lambda v: torch.as_tensor(np.asarray(v, dtype=np.int32), device=device)  # noqa: E731
        f64 = lambda v: torch.as_tensor(np.asarray(v, dtype=np.float64), device=device)  # noqa: E731
        ca, ct = csr_matrix(a), csr_matrix(a).T.tocsr()
        ca.sort_indices()
        ct.sort_indices()
        self.csr = (i32(ca.indptr), i32(ca.indices), f64(ca.data), i32(ct.indptr), i32(ct.indices), f64(ct.data))
        self.prow32, self.pcol32 = i32(patch[0]), i32(patch[1])


def fused_certificate(tpl: _Template, deltas, x, y, c, lower, upper, rhs, neq, row_group, col_group, table):
    """``certificate`` in one launch of the native kernel
    (``fbalp_scaled_certificate``): ``row_group`` / ``col_group`` int32
    group indices into the per-environment scale ``table``."""
    E = x.shape[0]
    dev = x.device
    out = torch.empty(3, E, dtype=torch.float64, device=dev)
    lib = N.load()
    p = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
    ap, ai, av, tp, ti, tv = tpl.csr
    npatch = 0 if deltas is None else int(deltas.shape[1])
    args = [x, y, c, lower, upper, rhs, table]
    if any(not t.is_contiguous() for t in args) or (deltas is not None and not deltas.is_contiguous()):
        raise ValueError("certificate inputs must be contiguous")
    N.check(lib.fbalp_scaled_certificate(
        E, tpl.m, tpl.n, int(neq), p(ap), p(ai), p(av), p(tp), p(ti), p(tv), npatch,
        p(tpl.prow32) if npatch else None, p(tpl.pcol32) if npatch else None, p(deltas) if npatch else None,
        p(x), p(y), p(c), p(lower), p(upper), p(rhs), p(row_group), p(col_group), int(table.shape[1]),
        p(table), p(out[0]), p(out[1]), p(out[2]),
        ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))
    return out[0], out[1], out[2]


def certificate(tpl: _Template, deltas, x, y, c, lower, upper, rhs, neq, row_scale, col_scale):
    """Per-environment certificate of the ORIGINAL (unscaled) LP from a
    solution of the scaled one: ``primal`` = max |equality residual|, max
    positive inequality residual and bound violation; ``dual`` = max positive
    inequality dual and wrong-signed reduced cost on infinite bounds;
    ``gap`` = (sum |d (x - active bound)| + sum |y_ub slack|) / max(1,
    |c.x|) (the formulas of ``src/gpu_block_lp.py:52-132``).  All inputs are
    ``(E, .)`` tensors of the scaled LP; ``row_scale`` / ``col_scale`` map
    original rows / columns to scaled ones."""
    act = (tpl.A @ x.T.contiguous()).T
    aty = (tpl.AT @ y.T.contiguous()).T
    if deltas is not None and deltas.shape[1]:
        act = act.index_add(1, tpl.prow, deltas * x[:, tpl.pcol])
        aty = aty.index_add(1, tpl.pcol, deltas * y[:, tpl.prow])
    res = act - rhs
    prim_rows = torch.cat([res[:, :neq].abs(), res[:, neq:].clamp_min(0.0)], dim=1) / row_scale
    bnd = torch.maximum(lower - x, x - upper).clamp_min(0.0)
    bnd = torch.where(torch.isfinite(bnd), bnd, torch.zeros_like(bnd)) / col_scale
    primal = torch.maximum(prim_rows.amax(1), bnd.amax(1))
    d = c - aty
    dv = d * col_scale
    yv_ub = y[:, neq:] * row_scale[:, neq:]
    dual = torch.maximum(yv_ub.clamp_min(0.0).amax(1) if yv_ub.shape[1] else torch.zeros_like(primal),
                         torch.maximum(torch.where(torch.isinf(lower), dv, torch.zeros_like(dv)).clamp_min(0.0).amax(1),
                                       torch.where(torch.isinf(upper), -dv, torch.zeros_like(dv)).clamp_min(0.0).amax(1)))
    target = torch.where(d >= 0.0, lower, upper)
    comp = torch.where(torch.isfinite(target), (d * (x - target)).abs(), torch.zeros_like(d)).sum(1)
    comp = comp + (y[:, neq:] * res[:, neq:]).abs().sum(1)
    gap = comp / (c * x).sum(1).abs().clamp_min(1.0)
    return primal, dual, gap


@dataclass
class CooperativeResult:
    ok: torch.Tensor               # bool (E,): every stage that ran succeeded
    stage: torch.Tensor            # int (E,): last successful stage (STAGE_*)
    fluxes: torch.Tensor           # (E, n_fluxes) the chosen stage's fluxes (original units)
    nu: torch.Tensor               # (E,) coexistence growth of the chosen stage
    coexistence: torch.Tensor      # (E,) stage-1 optimum (clamped at 0)
    aggregate: torch.Tensor        # (E,) live objective of the stage-2 choice
    objective_values: torch.Tensor  # (E, S) per-member objective values of ``fluxes``
    stages: dict                   # stage name -> dict(status, iterations, primal, dual, gap, certified)


@dataclass
class Scales:
    """Per-environment scalings of the transformed LP."""

    xbar: torch.Tensor       # (E,) largest floored biomass
    rho: torch.Tensor        # (E, S) X_s / Xbar
    rho_min: torch.Tensor    # (E,)
    rho_col: torch.Tensor    # (E, n_fluxes) rho of each flux column's member
    table: torch.Tensor      # (E, S + 3): rho_s..., 1/Xbar, rho_min, 1 (scale groups)


class StageAssembly:
    """Per-environment data of the transformed stage LPs as tensors on one
    device (the device the engine runs on; the CPU in the host tests)."""

    def __init__(self, structure: CommunityStructure, device):
        st = self.st = structure
        dev = self.device = torch.device(device)
        t = lambda a, dtype=None: torch.as_tensor(a, device=dev, dtype=dtype)  # noqa: E731
        self.g = t(st.global_objective, torch.float64)
        self.col_species = t(st.col_species)
        self.relax_cols = t(st.relax_cols)
        self.med_rows = t(st.medium_rows)
        self.med_reserved = t(st.medium_reserved)
        self.row_group1, self.row_group3 = t(st.row_group1), t(st.row_group3)
        self.col_group1, self.col_group3 = t(st.col_group1), t(st.col_group3)
        self.perf_cols = t(st.perf_cols)
        self.perf_species = t(st.col_species[st.perf_cols])
        self.var_cols = t(st.var_cols)
        self.var_stoich = t(st.var_stoich, torch.float64)
        self.growth_cols = t(st.growth_cols)
        self.objectives = [t(o, torch.float64) for o in st.objectives]
        self._c1 = None

    def scales(self, biomass) -> Scales:
        X = biomass.clamp_min(BIOMASS_FLOOR)
        xbar = X.amax(dim=1)
        rho = X / xbar[:, None]
        rho_min = rho.amin(dim=1)
        one = torch.ones_like(xbar)[:, None]
        table = torch.cat([rho, (1.0 / xbar)[:, None], rho_min[:, None], one], dim=1)
        return Scales(xbar, rho, rho_min, rho[:, self.col_species], table)

    def relaxed_lower(self, lower, max_crossfeed_uptake):
        """Cross-feeding relaxation of the exchange lower bounds
        (``_bounds`` ``:1010-1017``, Python scalar max: a NaN limit keeps the
        original bound)."""
        if not len(self.st.relax_cols):
            return lower
        lo = lower.clone()
        if len(self.st.relax_cols):
            limit = -abs(float(max_crossfeed_uptake))
            cap = torch.as_tensor([max(o, limit) for o in self.st.relax_orig.tolist()], dtype=lo.dtype,
                                  device=lo.device)
            lo[:, self.relax_cols] = torch.minimum(lo[:, self.relax_cols], cap)
        return lo

    def stage1(self, sc: Scales, lower, upper, medium, dt, growth_upper):
        """``(lw, uw, l1, u1, c1, rhs1, d1)``: scaled flux bounds, stage-1
        bounds / cost / right-hand side and the patched-entry deltas."""
        st = self.st
        E = sc.xbar.shape[0]
        f64 = dict(dtype=torch.float64, device=sc.xbar.device)
        lw, uw = lower * sc.rho_col, upper * sc.rho_col
        supply = medium[:, self.med_rows].clamp_min(0.0) / dt
        supply = torch.where(self.med_reserved, torch.full_like(supply, RESERVED_SUPPLY), supply)
        rhs1 = torch.cat([torch.zeros(E, st.neq + st.n_species, **f64), supply / sc.xbar[:, None]], dim=1)
        l1 = torch.cat([lw, torch.zeros(E, 1, **f64)], dim=1)
        u1 = torch.cat([uw, torch.full((E, 1), float(growth_upper), **f64)], dim=1)
        c1 = self._stage1_cost(E, sc.xbar.device)
        d1 = (sc.rho - 1.0).contiguous()
        return lw, uw, l1, u1, c1, rhs1, d1

    def _stage1_cost(self, E, device):
        """The stage-1 cost (-1 on nu), the same for every call: built once
        per batch size and shared (read-only)."""
        c1 = self._c1
        if c1 is None or c1.shape[0] != E or c1.device != torch.device(device):
            c1 = torch.zeros(E, self.st.n1, dtype=torch.float64, device=device)
            c1[:, self.st.nu] = -1.0
            self._c1 = c1
        return c1

    def stage2(self, sc: Scales, lw, uw, floor, nu_hi, cost=True):
        """Bounds with ``nu`` in ``[floor, nu_hi]`` and the live-objective
        cost (minimisation form, scaled; None unless ``cost``)."""
        E = sc.xbar.shape[0]
        f64 = dict(dtype=torch.float64, device=sc.xbar.device)
        l2 = torch.cat([lw, floor[:, None]], dim=1)
        u2 = torch.cat([uw, nu_hi[:, None]], dim=1)
        c2 = torch.cat([-self.g[None, :] / sc.rho_col, torch.zeros(E, 1, **f64)], dim=1) if cost else None
        return l2, u2, c2

    def aggregate(self, sc: Scales, x):
        return (self.g[None, :] * x[:, :self.st.n_fluxes] / sc.rho_col).sum(dim=1)

    def stage3(self, sc: Scales, l2, u2, rhs1, d1, aggregate, objective_fraction):
        """``(l3, u3, c3, rhs3, d3)`` of the parsimonious-exchange LP."""
        st = self.st
        E, A = sc.xbar.shape[0], st.n_aux
        f64 = dict(dtype=torch.float64, device=sc.xbar.device)
        l3 = torch.cat([l2, torch.zeros(E, A, **f64)], dim=1)
        u3 = torch.cat([u2, torch.full((E, A), float("inf"), **f64)], dim=1)
        c3 = torch.cat([torch.zeros(E, st.n1, **f64), sc.xbar[:, None].expand(E, A)], dim=1).contiguous()
        parts, deltas = [rhs1], [d1]
        if st.optimize_live_objectives:
            # the row exists when aggregate > 1e-9 (``:159``); otherwise its
            # coefficients are patched to zero (0 <= 0)
            active = aggregate > 1e-9
            parts.append(torch.where(active, -aggregate * objective_fraction * sc.rho_min,
                                     torch.zeros_like(aggregate))[:, None])
            g = self.g[self.perf_cols][None, :]
            ratio = sc.rho_min[:, None] / sc.rho[:, self.perf_species]
            deltas.append(torch.where(active[:, None], -g * (ratio - 1.0), g.expand(E, -1)))
        parts.append(torch.zeros(E, 2 * A, **f64))
        return l3, u3, c3, torch.cat(parts, dim=1), torch.cat(deltas, dim=1).contiguous()

    def transfers(self, x):
        """Smallest feasible scaled transfers ``t'_j = |stoich_j w_j|``."""
        return (self.var_stoich[None, :] * x[:, self.var_cols]).abs()

    def fluxes(self, sc: Scales, x):
        return x[:, :self.st.n_fluxes] / sc.rho_col

    def objective_values(self, fluxes):
        st = self.st
        return torch.stack([(fluxes[:, st.col_start[s]:st.col_start[s + 1]] * self.objectives[s]).sum(1)
                            for s in range(st.n_species)], dim=1)


class CooperativeSolver:
    """Cooperative community LP for a batch of environments on one GPU
    (``CooperativeCommunityFbaSolver`` with an exact LP backend).  Stage
    LPs of all environments are solved in one engine call each; every
    stage's solution must meet the engine's tolerances and pass the
    reference's certificate on the unscaled LP, otherwise the environment
    reports no solution (the exact-backend rule of ``:1747-1749, 1794-1796``,
    no CPU fallback).  Calls warm-start from the previous ones: ``warm_start
    = "extrapolate"`` (default) from the first-order extrapolation of the
    last two solutions, ``"previous"`` from the last one, both in the
    reference's units and rescaled to the new biomass; ``False`` solves
    cold."""

    def __init__(self, members, *, coexistence_fraction=0.99, objective_fraction=0.99,
                 maximum_coexistence_growth=None, optimize_live_objectives=False, parsimonious_exchange=True,
                 config: SolveConfig | None = None, options: EngineOptions | None = None, device=None,
                 warm_start="extrapolate", retry_iterations=400_000):
        if not torch.cuda.is_available():
            raise RuntimeError("a CUDA device is required (no CPU fallback)")
        self.structure = st = CommunityStructure(members, optimize_live_objectives=optimize_live_objectives)
        self.coexistence_fraction = float(np.clip(coexistence_fraction, 0.0, 1.0))
        self.objective_fraction = float(np.clip(objective_fraction, 0.0, 1.0))
        self.growth_upper = (DEFAULT_GROWTH_UPPER if maximum_coexistence_growth is None
                             else max(0.0, float(maximum_coexistence_growth)))
        self.optimize_live_objectives = bool(optimize_live_objectives)
        self.parsimonious = bool(parsimonious_exchange) and st.n_aux > 0
        if len(st.patch3[0] if self.parsimonious else st.patch1[0]) > N.MAX_PATCHES:
            raise ValueError(f"the cooperative LP needs more than {N.MAX_PATCHES} per-environment coefficients "
                             "(members + live-objective nonzeros)")
        # stage LPs of coupled communities take up to a few 10^4 iterations
        # cold (the parsimonious stage with binding shared pools)
        self.config = config or SolveConfig(max_iterations=100_000, fp32_max_iterations=100_000)
        if self.config.precision != "mixed" or not self.config.recentre:
            raise ValueError("environment-dependent coefficients need the re-centred mixed schedule")
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.options = options or EngineOptions(warps_per_block=32)
        self.engine1 = LPEngine([(st.template1, st.neq)], options=self.options, device=self.device)
        self.engine1.set_patches(0, *st.patch1)
        self.engine3 = None
        if self.parsimonious:
            self.engine3 = LPEngine([(st.template3, st.neq)], options=self.options, device=self.device)
            self.engine3.set_patches(0, *st.patch3)
        self.asm = StageAssembly(st, self.device)
        i32 = lambda v: torch.as_tensor(np.asarray(v, dtype=np.int32), device=self.device)  # noqa: E731
        self._rg32 = {"max_min": i32(st.row_group1), "aggregate_objective": i32(st.row_group1),
                      "parsimonious_exchange": i32(st.row_group3)}
        self._cg32 = {"max_min": i32(st.col_group1), "aggregate_objective": i32(st.col_group1),
                      "parsimonious_exchange": i32(st.col_group3)}
        self._tpl1 = _Template(st.template1, st.patch1, self.device)
        self._tpl3 = _Template(st.template3, st.patch3, self.device) if self.parsimonious else None
        if warm_start is True:
            warm_start = "previous"
        if warm_start not in (False, None, "previous", "extrapolate"):
            raise ValueError("warm_start must be False, 'previous' or 'extrapolate'")
        self.warm_start = warm_start or False
        self._prev2 = {}
        # environments stopped by the iteration cap get one more pass of
        # this many iterations, alone (0: no second pass)
        self.retry_iterations = int(retry_iterations)
        self._retry_engines = {}
        self.retries: dict = {}        # stage -> environments retried so far
        self.last_retried: dict = {}   # stage -> environments retried by the last call
        self.E = 0
        self._prev = {}

    # -- binding -------------------------------------------------------------
    def _bind(self, E):
        st, dev = self.structure, self.device
        f64 = dict(dtype=torch.float64, device=dev)
        self.E = E
        sid = np.zeros(E, np.int32)
        z1 = torch.zeros(E * st.n1, **f64)
        self.engine1.set_instances(sid, z1, z1, z1, torch.zeros(E * st.m1, **f64))
        if self.parsimonious:
            z3 = torch.zeros(E * st.n3, **f64)
            self.engine3.set_instances(sid, z3, z3, z3, torch.zeros(E * st.m3, **f64))
        self._prev = {}
        self._prev2 = {}

    def reset(self):
        """Forget the warm-start history."""
        self._prev = {}
        self._prev2 = {}

    def _warm(self, key, table, rg, cg):
        """The previous call's solution of stage ``key`` rescaled to the
        current scalings (x_w = D x_v, y_w = y_v / R)."""
        prev = self._prev.get(key)
        if prev is None or not self.warm_start:
            return None, None, None
        x, y, omega, old, _ = prev
        prev2 = self._prev2.get(key) if self.warm_start == "extrapolate" else None
        if prev2 is None:
            ratio = table / old                   # per scale group, then one gather per vector
            return (x * ratio[:, cg]).reshape(-1), (y / ratio[:, rg]).reshape(-1), omega
        # first-order extrapolation of the last two solutions in the
        # reference's units (v = w / D, y_v = R y_w), mapped to the current
        # scaling; the kernel projects onto the bounds and y_ub <= 0
        x2, y2, _, old2, _ = prev2
        xv = 2.0 * x / old[:, cg] - x2 / old2[:, cg]
        yv = 2.0 * y * old[:, rg] - y2 * old2[:, rg]
        return (xv * table[:, cg]).reshape(-1), (yv / table[:, rg]).reshape(-1), omega

    def _run(self, engine, key, table, rg, cg, lower, upper, cost, rhs, deltas, tpl, warm=None):
        E = self.E
        engine.set_instance_data(lower.reshape(-1), upper.reshape(-1), cost.reshape(-1), rhs.reshape(-1))
        engine.set_patch_values(deltas)
        wx, wy, wo = self._warm(key, table, rg, cg)
        if wx is None and warm is not None:
            wx, wy, wo = warm
        prev = self._prev.get(key)
        engine.set_iteration_hints(None if prev is None or not self.warm_start else prev[4])
        res: SolveResult = engine.solve(warm_x=wx, warm_y=wy, warm_omega=wo, config=self.config)
        n, m = cost.shape[1], rhs.shape[1]
        x = res.x[:E * n].view(E, n)
        y = res.y[:E * m].view(E, m)
        primal, dual, gap = fused_certificate(tpl, deltas, x, y, cost.contiguous(), lower.contiguous(),
                                              upper.contiguous(), rhs.contiguous(), self.structure.neq,
                                              self._rg32[key], self._cg32[key], table.contiguous())
        ok = (res.status == N.STATUS_OPTIMAL) & (primal <= PRIMAL_GATE) & (dual <= DUAL_GATE) & (gap <= GAP_GATE)
        # what a second pass for this stage's laggards needs (run by solve()
        # for the last stage, after the only host synchronisation of a call)
        self._last_run = (key, res, x, y, ok, primal, dual, gap, table, lower, upper, cost, rhs, deltas, tpl)
        if key in self._prev:
            self._prev2[key] = self._prev[key]
        self._prev[key] = (x, y, res.omega, table, res.iterations)
        info = dict(status=res.status, iterations=res.iterations, primal=primal, dual=dual, gap=gap,
                    certified=ok)
        return x, y, res, ok, info

    def _retry_laggards(self, key, res, x, y, ok, primal, dual, gap, table, lower, upper, cost, rhs, deltas, tpl):
        """Environments whose stage stopped at the iteration cap continue,
        alone, from their own iterates with ``retry_iterations`` more; their
        results (and certificate) replace the first pass's in place."""
        lag = (~ok) & (res.status == N.STATUS_ITERATION_LIMIT)
        idx = lag.nonzero().flatten()
        if idx.numel() == 0:
            return
        st = self.structure
        eng = self._retry_engines.get(key)
        if eng is None:
            stage3 = key == "parsimonious_exchange"
            eng = LPEngine([(st.template3 if stage3 else st.template1, st.neq)], options=self.options,
                           device=self.device)
            eng.set_patches(0, *(st.patch3 if stage3 else st.patch1))
            self._retry_engines[key] = eng
        k = int(idx.numel())
        sub = lambda t: t[idx].contiguous()  # noqa: E731
        lo, up, c, b, d, tb = (sub(t) for t in (lower, upper, cost, rhs, deltas, table))
        eng.set_instances(np.zeros(k, np.int32), lo.reshape(-1), up.reshape(-1), c.reshape(-1), b.reshape(-1))
        eng.set_patch_values(d)
        cfg = SolveConfig(**{**self.config.__dict__, "max_iterations": self.retry_iterations,
                             "fp32_max_iterations": self.retry_iterations})
        r2 = eng.solve(warm_x=sub(x).reshape(-1), warm_y=sub(y).reshape(-1), warm_omega=res.omega[idx].contiguous(),
                       config=cfg)
        n, m = x.shape[1], y.shape[1]
        x2, y2 = r2.x[:k * n].view(k, n), r2.y[:k * m].view(k, m)
        p2, d2, g2 = fused_certificate(tpl, d, x2, y2, c, lo, up, b, st.neq, self._rg32[key], self._cg32[key], tb)
        ok2 = (r2.status == N.STATUS_OPTIMAL) & (p2 <= PRIMAL_GATE) & (d2 <= DUAL_GATE) & (g2 <= GAP_GATE)
        x[idx], y[idx] = x2, y2
        res.status[idx] = r2.status
        res.iterations[idx] = res.iterations[idx] + r2.iterations
        res.omega[idx] = r2.omega
        res.metrics[idx] = r2.metrics
        primal[idx], dual[idx], gap[idx] = p2, d2, g2
        ok[idx] = ok2
        self.retries[key] = self.retries.get(key, 0) + k
        self.last_retried[key] = idx.tolist()

    # -- solve -----------------------------------------------------------------
    def solve(self, biomass, medium, dt, lower, upper, *, max_crossfeed_uptake=20.0) -> CooperativeResult:
        """Solve every environment's cooperative LPs.

        ``biomass`` (E, S) gDW/L; ``medium`` (E, K) concentrations of
        ``structure.metabolites`` (sorted ids); ``lower``/``upper`` (E,
        n_fluxes) live flux bounds of all members (member order);
        ``max_crossfeed_uptake`` as the reference's ``solve``."""
        st, dev, asm = self.structure, self.device, self.asm
        self.last_retried = {}
        if dt <= 0:
            raise ValueError("dt must be positive")
        biomass = torch.as_tensor(biomass, dtype=torch.float64, device=dev)
        medium = torch.as_tensor(medium, dtype=torch.float64, device=dev)
        lower = torch.as_tensor(lower, dtype=torch.float64, device=dev)
        upper = torch.as_tensor(upper, dtype=torch.float64, device=dev)
        E = biomass.shape[0]
        if biomass.shape != (E, st.n_species) or medium.shape != (E, len(st.metabolites)):
            raise ValueError("biomass / medium shapes do not match the community")
        if lower.shape != (E, st.n_fluxes) or upper.shape != (E, st.n_fluxes):
            raise ValueError("flux bounds do not match the community")
        lo = asm.relaxed_lower(lower, max_crossfeed_uptake)
        # one pass: false for lo > upper and for a NaN on either side
        if not bool((lo <= upper).all()):
            raise ValueError("invalid flux bounds")
        if E != self.E:
            self._bind(E)
        sc = asm.scales(biomass)
        lw, uw, l1, u1, c1, rhs1, d1 = asm.stage1(sc, lo, upper, medium, dt, self.growth_upper)
        stages = {}
        x1, y1, r1, ok1, stages["max_min"] = self._run(
            self.engine1, "max_min", sc.table, asm.row_group1, asm.col_group1, l1, u1, c1, rhs1, d1, self._tpl1)
        coexistence = torch.where(ok1, x1[:, st.nu].clamp_min(0.0), torch.zeros_like(sc.xbar))
        floor = coexistence * self.coexistence_fraction
        ok = ok1
        stage = torch.where(ok1, STAGE_MAX_MIN, STAGE_FAILED)
        chosen_x, chosen_y, chosen_r = x1, y1, r1
        nu_hi = coexistence if self.optimize_live_objectives else floor
        l2, u2, c2 = asm.stage2(sc, lw, uw, floor, nu_hi, cost=self.optimize_live_objectives)
        if self.optimize_live_objectives:
            x2, y2, r2, ok2, stages["aggregate_objective"] = self._run(
                self.engine1, "aggregate_objective", sc.table, asm.row_group1, asm.col_group1, l2, u2, c2, rhs1, d1,
                self._tpl1, warm=(x1.reshape(-1), y1.reshape(-1), r1.omega))
            ok = ok & ok2
            stage = torch.where(ok, STAGE_AGGREGATE, STAGE_FAILED)
            chosen_x, chosen_y, chosen_r = x2, y2, r2
        aggregate = asm.aggregate(sc, chosen_x)
        final_x = chosen_x
        if self.parsimonious:
            l3, u3, c3, rhs3, d3 = asm.stage3(sc, l2, u2, rhs1, d1, aggregate, self.objective_fraction)
            # without history: the chosen stage's solution with the smallest
            # feasible transfers
            x0 = torch.cat([chosen_x, asm.transfers(chosen_x)], dim=1)
            x0[:, st.nu] = torch.minimum(torch.maximum(x0[:, st.nu], floor), nu_hi)
            y0 = torch.cat([chosen_y, torch.zeros(E, st.m3 - st.m1, dtype=torch.float64, device=dev)], dim=1)
            x3, _, _, ok3, stages["parsimonious_exchange"] = self._run(
                self.engine3, "parsimonious_exchange", sc.table, asm.row_group3, asm.col_group3, l3, u3, c3, rhs3,
                d3, self._tpl3, warm=(x0.reshape(-1), y0.reshape(-1), chosen_r.omega))
            ok = ok & ok3
            stage = torch.where(ok, STAGE_PARSIMONIOUS, STAGE_FAILED)
            final_x = x3
        if self.retry_iterations > 0:
            # the last stage's laggards continue in a second pass, which
            # updates that stage's solution and flags in place; this is the
            # only host synchronisation of a call (laggards of an earlier
            # stage, not observed, fail closed)
            self._retry_laggards(*self._last_run)
            self._last_run = None
            ok = ok1
            if self.optimize_live_objectives:
                ok = ok & ok2
            if self.parsimonious:
                ok = ok & ok3
                stage = torch.where(ok, STAGE_PARSIMONIOUS, STAGE_FAILED)
            elif self.optimize_live_objectives:
                stage = torch.where(ok, STAGE_AGGREGATE, STAGE_FAILED)
                aggregate = asm.aggregate(sc, chosen_x)
            else:
                stage = torch.where(ok, STAGE_MAX_MIN, STAGE_FAILED)
                coexistence = torch.where(ok1, x1[:, st.nu].clamp_min(0.0), torch.zeros_like(sc.xbar))
                # the retried stage-1 solution is the chosen one
                aggregate = asm.aggregate(sc, chosen_x)
        fluxes = asm.fluxes(sc, final_x)
        fluxes = torch.where(ok[:, None], fluxes, torch.full_like(fluxes, float("nan")))
        return CooperativeResult(ok=ok, stage=stage, fluxes=fluxes, nu=final_x[:, st.nu], coexistence=coexistence,
                                 aggregate=aggregate, objective_values=asm.objective_values(fluxes), stages=stages)

    def close(self):
        for e in (self.engine1, self.engine3, *self._retry_engines.values()):
            if e is not None:
                e.close()


SECONDARY_POOL = 60       # shared extracellular metabolites outside the medium
SECONDARY_OFFSET = 100    # their ids: m100_e ... (medium ids stay below)


def synthetic_members(models, *, secondary=SECONDARY_POOL, seed=0):
    """Members of the synthetic community.  As in the reference, where every
    exchange reaction of an extracellular metabolite joins that
    metabolite's shared pool (``src/community_solver.py:775-790``), every
    exchange column is an exchange term (stoichiometry -1): a medium column
    exchanges its medium metabolite ``m{id:03d}_e``, every other exchange
    column one of ``secondary`` shared metabolites ``m{100+k:03d}_e`` drawn
    with a seeded generator.  The secondary metabolites are absent from the
    medium (supply 0), so a member can take one up only as far as others
    secrete it in the same step.  Original lower bounds are the default
    ones; the growth reaction is the biomass column (coefficient 1) and the
    live objective maximises it."""
    rng = np.random.default_rng(seed + 4242)
    out = []
    for m in models:
        medium = {int(c): int(i) for c, i in zip(m.medium_columns, m.medium_ids)}
        others = [c for c in range(m.n_exchange) if c not in medium]
        draw = rng.integers(0, secondary, len(others)) if secondary > 0 else np.empty(0, np.int64)
        ids = dict(medium)
        ids.update({c: SECONDARY_OFFSET + int(k) for c, k in zip(others, draw)})
        cols = range(m.n_exchange) if secondary > 0 else sorted(medium)
        out.append(Member(
            name=m.name, S=m.S, growth=int(m.biomass), objective=-np.asarray(m.cost, dtype=np.float64),
            direction="max", exchanges=tuple((f"m{ids[c]:03d}_e", int(c), -1.0) for c in cols),
            original_lower={int(c): float(m.lower[c]) for c in cols}))
    return out


class CooperativeCommunity:
    """All environments of a synthetic community stepped with the
    cooperative LP (the reference's ``fba_mode="cooperative"`` step,
    ``src/dfba_simulator.py:1757-1797`` with ``solve_cooperative_fba``
    ``:1245-1263``): Michaelis-Menten uptake bounds from the current medium,
    the staged cooperative solve with the shared pools, then the biomass
    Euler step (a member without a solution decays at -0.01 /h, ``:1790``)
    and the medium update with the beginning-of-step biomass."""

    def __init__(self, models, medium, biomass, *, dt=0.05, capacity=CARRYING_CAPACITY, max_uptake_rate=20.0,
                 maximum_coexistence_growth=0.005, optimize_live_objectives=False, parsimonious_exchange=True,
                 config: SolveConfig | None = None, options: EngineOptions | None = None, device=None,
                 warm_start="extrapolate"):
        self.device = dev = torch.device(device) if device is not None else torch.device("cuda")
        self.models = models
        self.dt = float(dt)
        self.capacity = float(capacity)
        self.max_uptake_rate = float(max_uptake_rate)
        self.solver = CooperativeSolver(
            synthetic_members(models), maximum_coexistence_growth=maximum_coexistence_growth,
            optimize_live_objectives=optimize_live_objectives, parsimonious_exchange=parsimonious_exchange,
            config=config, options=options, device=dev, warm_start=warm_start)
        st = self.solver.structure
        self.medium = torch.as_tensor(medium, dtype=torch.float64, device=dev).clone()
        self.biomass = torch.as_tensor(biomass, dtype=torch.float64, device=dev).clone()
        self.E = self.medium.shape[0]
        self.base_lower = torch.as_tensor(np.concatenate([m.lower for m in models]), device=dev)
        self.upper = torch.as_tensor(np.concatenate([m.upper for m in models]), device=dev)[None, :].expand(
            self.E, -1).contiguous()
        # medium column of every shared metabolite (-1: not in the medium,
        # supply 0)
        ids = [int(name[1:4]) for name in st.metabolites]
        self.met_ids = torch.as_tensor([i if i < SECONDARY_OFFSET else -1 for i in ids], device=dev)
        self._in_medium = self.met_ids >= 0
        self.mm = []
        for s, m in enumerate(models):
            cols = st.col_start[s] + np.asarray(m.medium_columns, dtype=np.int64)
            self.mm.append(dict(
                cols=torch.as_tensor(cols, device=dev), ids=torch.as_tensor(m.medium_ids, device=dev),
                vmax=torch.as_tensor(m.vmax, device=dev)[None, :], km=torch.as_tensor(m.km, device=dev)[None, :],
                orig=torch.as_tensor(m.lower[m.medium_columns], device=dev)[None, :],
                ub=torch.as_tensor(m.upper[m.medium_columns], device=dev)[None, :]))
        self.growth_cols = torch.as_tensor(st.growth_cols, device=dev)
        self.step_index = 0
        self.result: CooperativeResult | None = None
        self._lower = None

    def shared_medium(self):
        """Concentrations of the shared metabolites (``structure.metabolites``
        order); secondary metabolites are not in the medium."""
        out = torch.zeros(self.E, len(self.solver.structure.metabolites), dtype=torch.float64, device=self.device)
        out[:, self._in_medium] = self.medium[:, self.met_ids[self._in_medium]]
        return out

    def live_bounds(self):
        """Flux lower bounds after the Michaelis-Menten uptake update (one
        buffer: only the medium exchange columns change between steps)."""
        if self._lower is None:
            self._lower = self.base_lower[None, :].repeat(self.E, 1)
        lower = self._lower
        total = self.biomass.clamp_min(1e-6).sum(dim=1, keepdim=True)
        for mm in self.mm:
            lower[:, mm["cols"]] = uptake_lower(self.medium[:, mm["ids"]], total, self.dt, mm)
        return lower

    def step(self) -> CooperativeResult:
        res = self.solver.solve(self.biomass, self.shared_medium(), self.dt, self.live_bounds(), self.upper,
                                max_crossfeed_uptake=self.max_uptake_rate)
        self.integrate(res)
        self.result = res
        return res

    def integrate(self, res: CooperativeResult):
        ok = res.ok[:, None]
        flux = torch.where(ok, res.fluxes, torch.zeros_like(res.fluxes))
        mu = torch.where(ok, flux[:, self.growth_cols], torch.full_like(self.biomass, -0.01))
        X0 = self.biomass.clone()
        self.biomass.copy_(euler_biomass(self.biomass, mu, self.capacity, self.dt))
        delta = torch.zeros_like(self.medium)
        for s, mm in enumerate(self.mm):
            delta.index_add_(1, mm["ids"], flux[:, mm["cols"]] * X0[:, s:s + 1] * self.dt)
        self.medium.copy_(torch.clamp(self.medium + delta, min=0.0))
        self.step_index += 1

    def close(self):
        self.solver.close()
