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
