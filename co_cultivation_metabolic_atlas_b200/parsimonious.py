"""Parsimonious second stage of the FBA dFBA step (opt-in tie-break).

The growth-maximising FBA LPs of the community have degenerate optimal
faces: with growth at its optimum the exchange fluxes can move over a whole
face, so two exact solvers may return different fluxes and the simulated
medium drifts apart.  The reference resolves the same ambiguity in its
cooperative LP with a parsimonious exchange stage (minimise the summed
absolute exchange fluxes at the chosen growth,
``_assemble_parsimonious_exchange_lp``, ``src/community_solver.py:116-204``).
Here each species' FBA step gets that second stage:

    min  sum_j w_j t_j              over the exchange columns j
    s.t. S v = 0
         v_j - t_j <= 0,  -v_j - t_j <= 0
         l <= v <= u,  v_growth >= 0.99 mu*  (mu* the stage-1 optimum)
         0 <= t_j <= max(|l_j|, |u_j|)

with seeded weights ``w_j = 10^U[0, 1]`` per species: distinct generic
weights make the optimal exchange fluxes unique (equal weights leave ties
between exchange routes of equal length), so every exact solver returns the
same fluxes and the trajectories can be compared.  Measured with the CPU
restatement of the engine's re-centred PDHG on the weight-conserving
community: growth held within 1e-6 of its optimum leaves a sliver of a
feasible set on which first-order iterations stall (primal residual ~2e-5
after 6e4 iterations), and weights within 10 % of each other leave nearly
tied vertices (some LPs miss 6e4 iterations); a 1 % growth relaxation (the
reference's stage-3 objective fraction plays this role) and weights spread
over a decade certify every probed LP in 9-12 thousand iterations.  Column
order ``[v | t]``, rows ``[S; (E, -I); (-E, -I)]`` (equalities first).
"""

from __future__ import annotations

import numpy as np
from scipy.sparse import csr_matrix, hstack, identity, vstack

GROWTH_RELAXATION = 1e-2   # relative slack of the stage-1 growth in stage 2
GROWTH_FLOOR_ABS = 1e-9    # absolute slack (growth near zero)


def exchange_weights(model, species_index: int) -> np.ndarray:
    """The seeded exchange weights of one species (``n_exchange``)."""
    rng = np.random.default_rng(7001 + int(species_index))
    return 10.0 ** rng.random(model.n_exchange)


def stage_matrix(model):
    """``[S 0; E -I; -E -I]`` (rows ``m + 2 n_exchange``, equalities first)."""
    S = csr_matrix(model.S)
    m, n = S.shape
    k = model.n_exchange
    E = csr_matrix((np.ones(k), (np.arange(k), np.arange(k))), shape=(k, n))
    neg = -identity(k, format="csr")
    a = vstack([hstack([S, csr_matrix((m, k))]), hstack([E, neg]), hstack([-E, neg])]).tocsr()
    a.sum_duplicates()
    a.eliminate_zeros()
    a.sort_indices()
    return a


def stage_bounds(model, lower, upper, growth):
    """Stage-2 bounds of a batch: ``lower``/``upper`` (E, n) stage-1 bounds,
    ``growth`` (E,) stage-1 growth fluxes -> (E, n + k) lower and upper."""
    lower = np.atleast_2d(lower)
    upper = np.broadcast_to(upper, lower.shape)
    k = model.n_exchange
    lo = np.concatenate([lower, np.zeros((lower.shape[0], k))], axis=1)
    up = np.concatenate([upper, np.maximum(np.abs(lower[:, :k]), np.abs(upper[:, :k]))], axis=1)
    b = model.biomass
    lo[:, b] = np.maximum(lower[:, b], np.asarray(growth) * (1.0 - GROWTH_RELAXATION) - GROWTH_FLOOR_ABS)
    lo[:, b] = np.minimum(lo[:, b], up[:, b])
    return lo, up


def stage_cost(model, species_index: int) -> np.ndarray:
    return np.concatenate([np.zeros(model.S.shape[1]), exchange_weights(model, species_index)])
