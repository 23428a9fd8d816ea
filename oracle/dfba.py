"""dFBA coupling restated on the CPU (test infrastructure only).

Restates, for the synthetic community workload, the parts of the reference
simulator that turn a medium state into LP bounds and LP fluxes into the next
state:

* uptake bounds -- ``set_uptake_constraints`` (``src/dfba_simulator.py:
  640-667``): ``v_kin = v_max C/(K_m + C)``; ``v_phys = min(C/(sum_s
  max(1e-6, X_s) dt), 10 v_max)``; ``lb = min(0, max(-min(v_kin, v_phys),
  orig_lb))`` rounded to 6 decimals (``_safe_lb``, ``:553-563``).
* biomass -- ``update_biomass`` (``:1294-1324``) without the pH model (the
  synthetic medium has no proton balance): ``mu = clip(mu, -0.5, 2.0)``;
  ``dX = mu X (1 - sum X / K if mu > 0 else 1) dt``; ``X = clip(X + dX, 0, K)``.
* medium -- ``_update_environment`` (``:1326-1435``) for plain exchanged
  metabolites: ``C = max(0, C + sum_s v_s X_s dt)`` using the beginning-of-step
  biomass (``integration_biomass``, ``:1680-1683, 1797``).
* step order (``:1757-1797``): bounds from the current state -> LPs ->
  biomass update -> medium update.

The carrying capacity defaults to the reference's 20 gDW/L
(``src/dfba_simulator.py:104``).
"""

from __future__ import annotations

import numpy as np

CARRYING_CAPACITY = 20.0


def uptake_lower_bounds(model, medium, biomass, dt):
    """Per-environment lower bounds of one species (shape ``(E, n)``)."""
    medium = np.atleast_2d(np.asarray(medium, float))
    biomass = np.atleast_2d(np.asarray(biomass, float))
    E = medium.shape[0]
    lower = np.repeat(model.lower[None, :], E, axis=0)
    conc = medium[:, model.medium_ids]                       # (E, k)
    vmax = model.vmax[None, :]
    km = model.km[None, :]
    v_kin = vmax * conc / (km + conc)
    total = np.maximum(1e-6, biomass).sum(axis=1, keepdims=True)
    v_phys = np.minimum(conc / (total * dt), vmax * 10.0)
    limit = np.minimum(v_kin, v_phys)
    orig = model.lower[model.medium_columns][None, :]
    lb = np.minimum(0.0, np.maximum(-limit, orig))
    lb = np.minimum(lb, model.upper[model.medium_columns][None, :])
    lower[:, model.medium_columns] = np.round(lb, 6)
    return lower


def update_biomass(biomass, mu, dt, capacity=CARRYING_CAPACITY):
    """Euler biomass step for all species of all environments (``(E, S)``)."""
    mu = np.clip(mu, -0.5, 2.0)
    total = biomass.sum(axis=1, keepdims=True)
    cap = np.maximum(0.0, 1.0 - total / capacity)
    dX = mu * biomass * np.where(mu > 0, cap, 1.0) * dt
    return np.clip(biomass + dX, 0.0, capacity)


def update_medium(medium, models, fluxes, biomass0, dt):
    """Euler medium step: ``fluxes[s]`` is ``(E, n_s)``; ``biomass0`` the
    beginning-of-step biomass ``(E, S)``."""
    delta = np.zeros_like(medium)
    for s, mdl in enumerate(models):
        v = fluxes[s][:, mdl.medium_columns]                 # (E, k)
        contrib = v * biomass0[:, s:s + 1] * dt
        np.add.at(delta, (slice(None), mdl.medium_ids), contrib)
    return np.maximum(0.0, medium + delta)


def step(models, medium, biomass, dt, solve):
    """One dFBA step.  ``solve(species, lower)`` returns ``(status, mu, x)``
    arrays for all environments of that species (x of shape ``(E, n)``)."""
    fluxes, mus = [], []
    for s, mdl in enumerate(models):
        lower = uptake_lower_bounds(mdl, medium, biomass, dt)
        status, mu, x = solve(s, lower)
        if np.any(status != 0):
            raise RuntimeError("an LP was not solved; no fallback")
        fluxes.append(x)
        mus.append(mu)
    mu = np.stack(mus, axis=1)
    biomass0 = biomass.copy()
    biomass = update_biomass(biomass, mu, dt)
    medium = update_medium(medium, models, fluxes, biomass0, dt)
    return medium, biomass, fluxes


def parsimonious_fluxes(model, species_index, lower, upper, growth):
    """The parsimonious second stage of one species' FBA LP restated with
    HiGHS (the reference's exact solver): minimise the weighted sum of
    absolute exchange fluxes (weights of ``parsimonious.exchange_weights``)
    with growth held at ``growth (1 - GROWTH_RELAXATION) - 1e-9``, through the split
    ``t_j >= v_j, t_j >= -v_j`` (the pattern of
    ``_assemble_parsimonious_exchange_lp``, ``src/community_solver.py:
    116-204``).  Returns ``(status, fluxes v)``."""
    from scipy.optimize import linprog
    from scipy.sparse import csr_matrix, hstack, identity, vstack

    from co_cultivation_metabolic_atlas_b200.parsimonious import (GROWTH_FLOOR_ABS, GROWTH_RELAXATION,
                                                                  exchange_weights)
    S = csr_matrix(model.S)
    m, n = S.shape
    k = model.n_exchange
    w = exchange_weights(model, species_index)
    pick = csr_matrix((np.ones(k), (np.arange(k), np.arange(k))), shape=(k, n))
    a_eq = hstack([S, csr_matrix((m, k))]).tocsr()
    a_ub = vstack([hstack([pick, -identity(k)]), hstack([-pick, -identity(k)])]).tocsr()
    lo = np.concatenate([lower, np.zeros(k)])
    up = np.concatenate([upper, np.maximum(np.abs(lower[:k]), np.abs(upper[:k]))])
    b = model.biomass
    lo[b] = min(max(lower[b], growth * (1.0 - GROWTH_RELAXATION) - GROWTH_FLOOR_ABS), up[b])
    res = linprog(np.concatenate([np.zeros(n), w]), A_eq=a_eq, b_eq=np.zeros(m), A_ub=a_ub,
                  b_ub=np.zeros(2 * k), bounds=np.column_stack([lo, up]), method="highs-ds")
    if res.status != 0:
        return res.status, None
    return 0, np.asarray(res.x[:n])
