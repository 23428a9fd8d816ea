"""Seeded synthetic flux-balance workloads.

The reference project solves FBA LPs built from curated genome-scale models
(``src/dfba_simulator.py:1061-1102`` builds ``max c.v s.t. S v = 0,
l <= v <= u`` from a COBRA model).  Those models do not ship with this package;
the workloads below are seeded synthetic stand-ins with the shapes and value
distributions of the batched-LP benchmark:

* ``species_matrix`` -- one stoichiometric matrix: ``n_exchange`` exchange
  columns with a single ``-1``; internal columns with 2-6 nonzeros in distinct
  uniformly drawn rows, magnitudes 1 (85 %), 2 (10 %), 0.5 (5 %) with random
  sign; one biomass column with ``biomass_nnz`` entries of magnitude
  lognormal(-1, 1), 90 % of them negative (consumed precursors).
* 30 % of internal reactions reversible ``[-1000, 1000]``, the rest
  ``[0, 1000]``; exchange bounds ``[-u, 1000]`` with ``u ~ U[0, 20]``.
* the objective maximises the biomass column (minimisation form ``-e_bio``,
  as ``src/dfba_simulator.py:1080`` passes ``-c``).

Column order is ``[exchange | internal | biomass]``.

With the generator as specified the internal reactions do not conserve
anything (random signs), so internal cycles can supply every biomass
precursor and the biomass optimum is set by the internal bounds, not by
uptake: every instance of a species has the same optimal value.
``conserved=True`` draws positive metabolite weights ``w ~ U[0.5, 2]`` and
rescales one entry of every internal column so that ``w . column = 0``:
internal reactions then only move weight between metabolites, biomass
(which consumes weight) must be paid for by uptake, and the per-instance
uptake caps set the optimal value (``binding_species_workload``, a parity
family whose objectives differ per instance).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
from scipy.sparse import coo_matrix, csr_matrix

BOUND = 1000.0


@dataclass
class SpeciesModel:
    """One synthetic species: matrix, default bounds, objective."""

    name: str
    S: csr_matrix
    lower: np.ndarray
    upper: np.ndarray
    cost: np.ndarray            # minimisation objective (-e_biomass)
    n_exchange: int
    biomass: int                # column index of the biomass reaction
    anchor: np.ndarray | None = None  # a feasible flux of the default bounds (scale workload)
    medium_columns: np.ndarray = field(default_factory=lambda: np.empty(0, np.int64))
    medium_ids: np.ndarray = field(default_factory=lambda: np.empty(0, np.int64))
    vmax: np.ndarray = field(default_factory=lambda: np.empty(0))
    km: np.ndarray = field(default_factory=lambda: np.empty(0))

    @property
    def shape(self):
        return self.S.shape


def species_matrix(m: int, n: int, *, n_exchange: int = 200, biomass_nnz: int = 60,
                   seed: int = 0, name: str = "species", conserved: bool = False):
    """Build one synthetic species (see module docstring; ``conserved``:
    internal reactions balanced against positive metabolite weights)."""
    if n < n_exchange + 2 or m < 6 or biomass_nnz > m:
        raise ValueError("species dimensions too small")
    rng = np.random.default_rng(seed)
    n_int = n - n_exchange - 1
    rows = [rng.integers(0, m, n_exchange)]
    cols = [np.arange(n_exchange)]
    vals = [np.full(n_exchange, -1.0)]
    counts = rng.integers(2, 7, n_int)
    total = int(counts.sum())
    r_int = np.empty(total, np.int64)
    pos = 0
    for k in counts:
        r_int[pos:pos + k] = rng.choice(m, int(k), replace=False)
        pos += k
    u = rng.random(total)
    mag = np.where(u < 0.85, 1.0, np.where(u < 0.95, 2.0, 0.5))
    sgn = np.where(rng.random(total) < 0.5, -1.0, 1.0)
    if conserved:
        # per column, the entry of the heaviest metabolite balances the rest;
        # a balancing value below 0.05 in magnitude (a near-cancelling draw)
        # flips the sign of another entry first
        weight = conservation_weights(m, seed)
        v = mag * sgn
        pos = 0
        for k in counts:
            k = int(k)
            wr = weight[r_int[pos:pos + k]]
            vs = v[pos:pos + k]
            j = int(np.argmax(wr))
            q = (j + 1) % k
            for _ in range(2):
                vj = -(float(np.dot(wr, vs)) - wr[j] * vs[j]) / wr[j]
                if abs(vj) >= 0.05:
                    break
                vs[q] = -vs[q]
            vs[j] = vj
            pos += k
        mag, sgn = np.abs(v), np.sign(v)
    rows.append(r_int)
    cols.append(np.repeat(np.arange(n_exchange, n_exchange + n_int), counts))
    vals.append(mag * sgn)
    rb = rng.choice(m, biomass_nnz, replace=False)
    vb = rng.lognormal(-1.0, 1.0, biomass_nnz) * np.where(rng.random(biomass_nnz) < 0.9, -1.0, 1.0)
    rows.append(rb)
    cols.append(np.full(biomass_nnz, n - 1))
    vals.append(vb)
    S = coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                   shape=(m, n)).tocsr()
    S.sum_duplicates()
    S.eliminate_zeros()
    S.sort_indices()
    lower = np.zeros(n)
    upper = np.full(n, BOUND)
    reversible = rng.random(n_int) < 0.3
    lower[n_exchange:n_exchange + n_int][reversible] = -BOUND
    lower[:n_exchange] = -rng.uniform(0.0, 20.0, n_exchange)
    cost = np.zeros(n)
    cost[n - 1] = -1.0
    return SpeciesModel(name=name, S=S, lower=lower, upper=upper, cost=cost,
                        n_exchange=n_exchange, biomass=n - 1), rng


def conservation_weights(m: int, seed: int = 0) -> np.ndarray:
    """The positive metabolite weights ``w`` of ``species_matrix(...,
    conserved=True)`` with the same ``m`` and ``seed``: ``w . S[:, j] = 0``
    for every internal column ``j``."""
    return np.random.default_rng(seed + 15485863).uniform(0.5, 2.0, m)


def exchange_batch(model: SpeciesModel, count: int, *, seed: int = 1):
    """Per-instance bounds for the single-species batch: exchange lower
    bounds ``-u_i`` with ``u_i ~ U[0, 20]`` drawn independently per instance.

    Returns ``(lower, upper)`` arrays of shape ``(count, n)``.
    """
    rng = np.random.default_rng(seed)
    n = model.S.shape[1]
    lower = np.repeat(model.lower[None, :], count, axis=0)
    upper = np.repeat(model.upper[None, :], count, axis=0)
    lower[:, :model.n_exchange] = -rng.uniform(0.0, 20.0, (count, model.n_exchange))
    return lower, upper


def single_species_workload(count: int = 256, *, m: int = 1200, n: int = 2600, seed: int = 0):
    """The 256-instance single-species FBA batch (1,200 x 2,600)."""
    model, _ = species_matrix(m, n, seed=seed, name="single")
    lower, upper = exchange_batch(model, count, seed=seed + 1)
    return model, lower, upper


def binding_species_workload(count: int = 256, *, m: int = 1200, n: int = 2600, seed: int = 0):
    """The single-species batch on a weight-conserving species: uptake caps
    ``u_i ~ U[0, 20]`` bind, so the optimal value differs per instance."""
    model, _ = species_matrix(m, n, seed=seed, name="binding", conserved=True)
    lower, upper = exchange_batch(model, count, seed=seed + 1)
    return model, lower, upper


COMMUNITY_SIZES = ((950, 1800), (1400, 2700), (1100, 2200))
# Seed of the full-size community used for the cooperative (max-min growth)
# LP: the lowest seed whose three members can all grow at default bounds
# (seed 0's first member cannot, which pins the max-min growth at 0 and
# makes every cooperative LP's optimum the zero flux).
COOPERATIVE_SEED = 11
# Seed of the weight-conserving (uptake-binding) community: the lowest seed
# whose three conserved members all grow at the initial media.
BINDING_SEED = 2
LARGE_SIZES = ((3000, 6000), (2500, 5200), (3400, 6800))
MEDIUM_SIZE = 40
MEDIUM_PER_SPECIES = 25


def community_models(sizes=COMMUNITY_SIZES, *, seed: int = 0, n_medium: int = MEDIUM_SIZE,
                     per_species: int = MEDIUM_PER_SPECIES, fixed_fraction: float = 0.0,
                     duplicate_fraction: float = 0.0, conserved: bool = False):
    """Three species sharing an ``n_medium``-metabolite medium.

    Each species maps ``per_species`` of its exchange columns onto a random
    subset of the medium metabolites, with Michaelis-Menten parameters
    ``v_max ~ U[5, 20]`` and ``K_m ~ U[0.01, 1]``.  The other exchange columns
    keep the fixed bounds drawn by ``species_matrix``.  ``fixed_fraction`` of
    the non-medium exchange bounds are fixed (``l = u``) and
    ``duplicate_fraction`` of the reversible internal reactions receive a
    parallel duplicate column (the scale/degeneracy stress workload).
    ``conserved`` builds weight-conserving species (module docstring), whose
    growth is limited by the Michaelis-Menten uptake of the medium.

    Fixed exchange values drawn independently (``U[0, 2]``) make most draws
    infeasible (measured: with secretions fixed two of the three large
    species have no feasible flux, with uptakes fixed the third), and a
    batch of infeasible LPs measures nothing.  The fixed values are
    therefore taken from a feasible flux: ``anchor`` = the optimum of the
    species' network for a seeded random objective (HiGHS, default bounds),
    scaled so that its fixed exchange values lie in ``[-2, 2]`` (the scaled
    flux stays feasible because the bounds contain 0); the value magnitudes
    keep the ``[0, 2]`` range, their signs are the network's.
    """
    rng = np.random.default_rng(seed + 7919)
    models = []
    for k, (m, n) in enumerate(sizes):
        dup = 0
        if duplicate_fraction > 0:
            # Reserve columns for duplicates so that the total column count
            # stays at n: build a narrower matrix, then append duplicates.
            dup = int(round(duplicate_fraction * 0.3 * (n - 201)))
        model, _ = species_matrix(m, n - dup, seed=seed * 101 + k, name=f"species{k}", conserved=conserved)
        if dup:
            reversible = np.flatnonzero(model.lower[model.n_exchange:model.biomass] < 0) + model.n_exchange
            pick = rng.choice(reversible, dup, replace=False)
            S = model.S.tocsc()
            from scipy.sparse import hstack
            body = hstack([S[:, :model.biomass], S[:, pick], S[:, model.biomass:]]).tocsr()
            body.sort_indices()
            lower = np.concatenate([model.lower[:model.biomass], model.lower[pick], model.lower[model.biomass:]])
            upper = np.concatenate([model.upper[:model.biomass], model.upper[pick], model.upper[model.biomass:]])
            cost = np.zeros(body.shape[1])
            cost[-1] = -1.0
            model = SpeciesModel(name=model.name, S=body, lower=lower, upper=upper, cost=cost,
                                 n_exchange=model.n_exchange, biomass=body.shape[1] - 1)
        cols = rng.choice(model.n_exchange, per_species, replace=False)
        cols.sort()
        ids = rng.choice(n_medium, per_species, replace=False)
        model.medium_columns = cols.astype(np.int64)
        model.medium_ids = ids.astype(np.int64)
        model.vmax = rng.uniform(5.0, 20.0, per_species)
        model.km = rng.uniform(0.01, 1.0, per_species)
        model.lower[cols] = -BOUND
        if fixed_fraction > 0:
            others = np.setdiff1d(np.arange(model.n_exchange), cols)
            fixed = rng.choice(others, int(round(fixed_fraction * len(others))), replace=False)
            flux = _feasible_flux(model, rng)
            peak = float(np.abs(flux[fixed]).max(initial=0.0))
            scale = rng.uniform(0.0, 2.0) / peak if peak > 0 else 0.0
            model.anchor = flux * min(1.0, scale)
            model.lower[fixed] = model.anchor[fixed]
            model.upper[fixed] = model.anchor[fixed]
        models.append(model)
    return models


def _feasible_flux(model: SpeciesModel, rng) -> np.ndarray:
    """A vertex flux of ``S v = 0`` within the model's bounds that optimises
    a random objective (HiGHS interior point with crossover)."""
    from scipy.optimize import linprog
    objective = rng.uniform(-1.0, 1.0, model.S.shape[1])
    res = linprog(objective, A_eq=model.S, b_eq=np.zeros(model.S.shape[0]),
                  bounds=np.column_stack([model.lower, model.upper]), method="highs-ipm")
    if res.status != 0:
        raise RuntimeError("species network has no feasible flux")
    return np.clip(np.asarray(res.x), model.lower, model.upper)


def scale_batch(models, count: int, *, mix=(0.5, 0.3, 0.2), seed: int = 0):
    """An uneven batch of the scale workload: ``count`` instances split over
    the species by ``mix``; each instance draws its free exchange lower
    bounds ``-u`` with ``u ~ U[0, 20]`` (widened to contain the species'
    anchor flux, so every instance stays feasible).  Returns the species id
    of every instance and per-species ``(lower, upper)`` arrays."""
    rng = np.random.default_rng(seed + 31337)
    sizes = np.floor(np.asarray(mix, float) / np.sum(mix) * count).astype(int)
    sizes[0] += count - sizes.sum()
    species_id = np.repeat(np.arange(len(models), dtype=np.int32), sizes)
    bounds = []
    for s, mdl in enumerate(models):
        k = int(sizes[s])
        lower = np.repeat(mdl.lower[None, :], k, axis=0)
        free = np.flatnonzero((mdl.lower[:mdl.n_exchange] < mdl.upper[:mdl.n_exchange]))
        draw = -rng.uniform(0.0, 20.0, (k, len(free)))
        if mdl.anchor is not None:
            draw = np.minimum(draw, mdl.anchor[free][None, :])
        lower[:, free] = draw
        bounds.append((lower, np.repeat(mdl.upper[None, :], k, axis=0)))
    return species_id, bounds


def initial_environments(count: int, n_medium: int = MEDIUM_SIZE, n_species: int = 3, *, seed: int = 0):
    """Initial medium concentrations ``lognormal(0, 1)`` mM and biomass
    ``U[0.01, 0.1]`` gDW/L for ``count`` environments."""
    rng = np.random.default_rng(seed + 104729)
    medium = rng.lognormal(0.0, 1.0, (count, n_medium))
    biomass = rng.uniform(0.01, 0.1, (count, n_species))
    return medium, biomass
