"""The autotuner times every candidate launch shape on a seeded sample of a
batch, picks the fastest per certified LP, and caches its choice by the
workload's matrices and the device."""
import numpy as np
import pytest

from co_cultivation_metabolic_atlas_b200 import synthetic as syn
from oracle import dfba
from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="CUDA device required")]


def test_autotune_picks_a_certifying_shape_and_caches_it(tmp_path):
    import torch
    from co_cultivation_metabolic_atlas_b200.autotune import autotune
    from co_cultivation_metabolic_atlas_b200.engine import LPEngine
    models = syn.community_models()[:2]
    envs = 200
    medium, biomass = syn.initial_environments(envs, seed=4)
    mats = [(m.S, m.S.shape[0]) for m in models]
    sid = np.repeat(np.arange(2, dtype=np.int32), envs)
    lower = torch.as_tensor(np.concatenate([dfba.uptake_lower_bounds(m, medium, biomass, 0.05).ravel()
                                            for m in models]), device="cuda")
    upper = torch.as_tensor(np.concatenate([np.tile(m.upper, envs) for m in models]), device="cuda")
    cost = torch.as_tensor(np.concatenate([np.tile(m.cost, envs) for m in models]), device="cuda")
    eng = LPEngine(mats)
    co, _, _, _ = eng.layout(sid)
    eng.close()
    cache = tmp_path / "tune.json"
    opts, cfg, timings = autotune(mats, sid, lower, upper, cost, co, sample=400, warps=(8, 16), check_every=(64,),
                                  cache=cache)
    rows = [t for t in timings if "error" not in t]
    assert len(rows) == 4 and all(t["certified"] == 400 for t in rows)
    assert {t["kernel"] for t in rows} == {"pdhg_recentred_pair", "pdhg_recentred<staged>"}
    best = min(rows, key=lambda t: t["seconds_per_certified_lp"])
    assert (opts.warps_per_block, opts.pair_instances, cfg.check_every) == (best["warps_per_block"],
                                                                            best["pair_instances"], 64)
    # the cached choice is returned without timing again
    opts2, cfg2, timings2 = autotune(mats, sid, lower, upper, cost, co, sample=400, warps=(8, 16),
                                     check_every=(64,), cache=cache)
    assert (opts2, cfg2) == (opts, cfg) and timings2 == timings
    # and certifies the whole batch
    eng = LPEngine(mats, options=opts)
    eng.set_instances(sid, lower, upper, cost)
    res = eng.solve(config=cfg)
    assert int((res.status == 0).sum().item()) == 2 * envs
    eng.close()
