"""The learned warm start: trained on the engine's own rollouts (seeds
disjoint from the evaluated environments), it must cut PDHG iterations
against cold PDHG (the method without it) and never cost certification; its
first-step seed must beat a cold first step, and the trajectory it starts
must not lose later against one started cold."""
import numpy as np
import pytest

from co_cultivation_metabolic_atlas_b200 import synthetic as syn
from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="CUDA device required")]

ENVS = 256
STEPS = 6


def rollout(models, warm, learned=None, seed=7):
    import torch
    from co_cultivation_metabolic_atlas_b200.dfba import DeviceCommunity
    medium, biomass = syn.initial_environments(ENVS, seed=seed)
    com = DeviceCommunity(models, medium, biomass, warm_start=warm, learned=learned)
    iters, cert = [], 0
    for _ in range(STEPS):
        st = com.step()
        iters.append(st.iterations.float().mean().item())
        cert += int(st.certified.item())
    torch.cuda.synchronize()
    com.close()
    return np.array(iters), cert


@pytest.fixture(scope="module")
def trained():
    from co_cultivation_metabolic_atlas_b200 import train_warmstart as tw
    models = syn.community_models()
    data = tw.build_dataset(models, envs=ENVS, steps=8, seeds=[301, 302], log=lambda *_: None)
    ws, losses = tw.fit(models, data, epochs=6, batch=512, log=lambda *_: None)
    return models, ws, losses


def test_training_losses_decrease(trained):
    _, _, losses = trained
    assert losses[-1] < losses[0]


def test_learned_warm_start_gains_over_cold_pdhg(trained):
    models, ws, _ = trained
    it_l, cert_l = rollout(models, "learned", ws)
    it_c, cert_c = rollout(models, "cold")
    it_b, cert_b = rollout(models, "extrapolate")
    total = ENVS * 3 * STEPS
    assert cert_l == cert_c == cert_b == total  # every seed is driven to the same tolerances
    print(f"mean PDHG iterations per LP by step: learned {np.round(it_l, 1).tolist()}, "
          f"temporal base after a cold first step {np.round(it_b, 1).tolist()}, cold {np.round(it_c, 1).tolist()}")
    assert it_l.mean() <= 0.5 * it_c.mean()            # what the trained network gains over plain PDHG
    assert it_l[0] <= 0.8 * it_c[0]                    # its first-step seed beats a cold first step
    assert it_l[1:].mean() <= 1.05 * it_b[1:].mean()   # and the trajectory it starts does not lose later
