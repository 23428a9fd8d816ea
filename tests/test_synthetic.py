"""The seeded generator follows the workload's stated distributions."""
import numpy as np

from co_cultivation_metabolic_atlas_b200 import synthetic as syn


def test_single_species_structure():
    model, lower, upper = syn.single_species_workload(16)
    S = model.S.tocsc()
    m, n = S.shape
    assert (m, n) == (1200, 2600)
    ex = np.diff(S.indptr)[:200]
    assert np.all(ex == 1) and np.all(S.data[S.indptr[0]:S.indptr[200]] == -1.0)
    internal = np.diff(S.indptr)[200:n - 1]
    assert internal.min() >= 2 and internal.max() <= 6
    vals = np.abs(S[:, 200:n - 1].data)
    assert set(np.unique(vals)) <= {0.5, 1.0, 2.0}
    assert abs(np.mean(vals == 1.0) - 0.85) < 0.02
    assert np.diff(S.indptr)[n - 1] == 60
    assert np.mean(S[:, n - 1].data < 0) > 0.75
    rev = lower[0, 200:n - 1] < 0
    assert abs(rev.mean() - 0.3) < 0.03
    assert np.all(lower[:, :200] <= 0) and np.all(lower[:, :200] >= -20)
    assert not np.allclose(lower[0, :200], lower[1, :200])
    assert np.all(upper == 1000.0)
    assert model.cost[n - 1] == -1.0 and np.count_nonzero(model.cost) == 1


def test_community_structure():
    models = syn.community_models()
    assert [m.S.shape for m in models] == [(950, 1800), (1400, 2700), (1100, 2200)]
    for mdl in models:
        assert len(mdl.medium_columns) == 25 and len(set(mdl.medium_ids)) == 25
        assert mdl.medium_ids.max() < 40
        assert np.all((mdl.vmax >= 5) & (mdl.vmax <= 20)) and np.all((mdl.km >= 0.01) & (mdl.km <= 1))
    medium, biomass = syn.initial_environments(4096)
    assert medium.shape == (4096, 40) and biomass.shape == (4096, 3)
    assert biomass.min() >= 0.01 and biomass.max() <= 0.1


def test_large_species_with_fixed_and_duplicate_columns():
    models = syn.community_models(syn.LARGE_SIZES, fixed_fraction=0.2, duplicate_fraction=0.05)
    assert [m.S.shape for m in models] == [(3000, 6000), (2500, 5200), (3400, 6800)]
    for mdl in models:
        fixed = mdl.lower[:mdl.n_exchange] == mdl.upper[:mdl.n_exchange]
        assert abs(fixed.sum() - round(0.2 * (mdl.n_exchange - 25))) <= 1


def test_conserved_species_balances_every_internal_reaction():
    """``conserved=True``: every internal column is balanced against the
    positive metabolite weights, so biomass can only be paid for by uptake."""
    model, lower, upper = syn.binding_species_workload(4, m=300, n=650, seed=3)
    w = syn.conservation_weights(300, 3)
    S = model.S.tocsc()
    internal = S[:, model.n_exchange:model.biomass]
    np.testing.assert_allclose(w @ internal.toarray(), 0.0, atol=1e-12)
    counts = np.diff(S.indptr)
    assert counts[:model.n_exchange].tolist() == [1] * model.n_exchange
    assert counts[model.n_exchange:model.biomass].min() >= 2 and counts[model.biomass] == 60
    assert np.abs(internal.data).min() > 0.04
    # the biomass column consumes weight
    assert float(w @ S[:, model.biomass].toarray().ravel()) < 0


def test_uptake_binds_in_the_conserved_family():
    """The binding family's HiGHS optima differ per instance (uptake caps
    set them), unlike the specification's generator, where every instance
    of a species has the same optimum."""
    from oracle import highs
    model, lower, upper = syn.binding_species_workload(6, m=300, n=900, seed=3)
    res, _ = highs.solve_batch([model.S] * 6, list(lower), list(upper), [model.cost] * 6, workers=2)
    funs = np.array([r[1] for r in res])
    assert all(r[0] == 0 for r in res) and np.ptp(funs) > 1e-2 * np.abs(funs).max()
    spec, lo2, up2 = syn.single_species_workload(3, m=300, n=900, seed=3)
    res2, _ = highs.solve_batch([spec.S] * 3, list(lo2), list(up2), [spec.cost] * 3, workers=2)
    assert np.ptp([r[1] for r in res2]) < 1e-9
