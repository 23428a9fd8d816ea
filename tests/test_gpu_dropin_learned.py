"""The learned warm start through the drop-in: ``B200LPBackend(mode='mlp')``
with a ``RequestWarmStart`` trained on the engine's own rollouts (seeds
disjoint from the evaluated environments).  With ``linprog`` forbidden, the
first step's requests are seeded by the networks, the next step's by each
environment's temporal base; both need fewer PDHG iterations than cold
PDHG and certify the same rows with the same objectives.  A call that raises
leaves every environment's history as it was."""
import numpy as np
import pytest

from co_cultivation_metabolic_atlas_b200 import synthetic as syn
from oracle import dfba
from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="CUDA device required")]

ENVS = 48


@pytest.fixture(scope="module")
def trained():
    from co_cultivation_metabolic_atlas_b200.warmstart import fit_request_warm_start
    models = syn.community_models()
    ws, losses = fit_request_warm_start(models, envs=256, steps=6, seeds=[501, 502], epochs=15)
    return models, ws, losses


def requests(models, medium, biomass):
    reqs, ids = [], []
    for s, m in enumerate(models):
        lower = dfba.uptake_lower_bounds(m, medium, biomass, 0.05)
        zeros = np.zeros(m.S.shape[0])
        for e in range(medium.shape[0]):
            reqs.append((m.cost, dict(A_eq=m.S, b_eq=zeros, bounds=np.column_stack([lower[e], m.upper]),
                                      method="highs-ds")))
            ids.append((s, e))
    return reqs, ids


def next_state(models, medium, biomass, rows):
    fluxes = [np.stack([rows[s * ENVS + e].x for e in range(ENVS)]) for s in range(len(models))]
    mu = np.stack([f[:, m.biomass] for f, m in zip(fluxes, models)], axis=1)
    return dfba.update_medium(medium, models, fluxes, biomass, 0.05), dfba.update_biomass(biomass, mu, 0.05)


def test_training_losses_decrease(trained):
    _, _, losses = trained
    assert all(ls[-1] < ls[0] for ls in losses)


def test_learned_warm_start_through_solve_batch(trained, forbid_cpu_optimizers):
    from co_cultivation_metabolic_atlas_b200.backend import B200LPBackend
    models, ws, _ = trained
    ws.reset()
    medium, biomass = syn.initial_environments(ENVS, seed=9)
    cold = B200LPBackend(mode="cold")
    learned = B200LPBackend(mode="mlp", warm_start_model=ws)
    its = {"cold": [], "mlp": []}
    for step in range(2):
        reqs, ids = requests(models, medium, biomass)
        rows_c = cold.solve_batch(reqs, environment_ids=ids)
        rows_l = learned.solve_batch(reqs, environment_ids=ids)
        assert ws.last_sources == (["network"] if step == 0 else ["temporal"]) * len(ids)
        assert all(r.success for r in rows_c) and all(r.success for r in rows_l)
        fc = np.array([r.fun for r in rows_c])
        fl = np.array([r.fun for r in rows_l])
        assert np.all(np.abs(fc - fl) <= 1e-6 * np.maximum(1.0, np.abs(fc)))
        its["cold"].append(np.mean([r.diagnostics["iterations"] for r in rows_c]))
        its["mlp"].append(np.mean([r.diagnostics["iterations"] for r in rows_l]))
        medium, biomass = next_state(models, medium, biomass, rows_l)
    print(f"mean PDHG iterations per LP, steps 0-1: cold {its['cold']}, learned {its['mlp']}")
    assert its["mlp"][0] <= 0.8 * its["cold"][0]   # the networks' seeds beat cold starts
    assert its["mlp"][1] <= 0.5 * its["cold"][1]   # the temporal base afterwards
    cold.close()
    learned.close()


def test_a_call_that_raises_does_not_advance_the_history(trained, forbid_cpu_optimizers):
    from co_cultivation_metabolic_atlas_b200.backend import B200LPBackend
    models, ws, _ = trained
    ws.reset()
    medium, biomass = syn.initial_environments(8, seed=21)
    reqs, ids = requests(models, medium, biomass)
    be = B200LPBackend(mode="mlp", warm_start_model=ws)
    be.solve_batch(reqs[:8], environment_ids=ids[:8])
    before = {env: [id(h[1]) for h in hist] for env, hist in ws._history.items()}
    eng = be._engine

    def broken(*_a, **_k):
        raise RuntimeError("device lost")
    eng.solve = broken
    with pytest.raises(RuntimeError):
        be.solve_batch(reqs[:8], environment_ids=ids[:8])
    after = {env: [id(h[1]) for h in hist] for env, hist in ws._history.items()}
    assert after == before and len(be.history) == 1
    be.close()
