"""The scale/degeneracy workload (three large species, fixed exchange
bounds, duplicated reversible columns): a cold batch, the same batch from the
learned warm start (request networks trained on cold solves of batches
drawn with other seeds) and a warm re-solve after perturbed bounds; every LP
is certified and both warm starts need fewer iterations than cold PDHG."""
import argparse

import pytest

from co_cultivation_metabolic_atlas_b200 import synthetic as syn
from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="CUDA device required")]


def test_scale_sweep_cold_learned_and_warm():
    import torch
    from co_cultivation_metabolic_atlas_b200 import sweep
    device = torch.device("cuda", 0)
    models = syn.community_models(syn.LARGE_SIZES, fixed_fraction=0.2, duplicate_fraction=0.05)
    args = argparse.Namespace(mix=[0.5, 0.3, 0.2], seed=0, autotune=False, cache=None)
    members = sweep.train_members(models, args, device, count=600, seeds=(101,), epochs=10)
    out = sweep.run(400, models, args, device, members)
    for phase in ("cold", "learned", "warm"):
        assert out[phase]["certified"] == 400, (phase, out[phase])
    print({p: out[p]["iterations"]["mean"] for p in ("cold", "learned", "warm")})
    assert out["learned"]["iterations"]["mean"] < out["cold"]["iterations"]["mean"]
    assert out["warm"]["iterations"]["mean"] < 0.5 * out["cold"]["iterations"]["mean"]
