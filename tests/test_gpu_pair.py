"""The paired re-centred kernel (two instances of a species per CTA, one
staged matrix, interleaved vectors) computes exactly what the
single-instance re-centred kernel computes: per instance the same operations
in the same order, so statuses, iteration counts, fluxes, duals and metrics
are equal bit for bit -- on cold and warm-started batches, across species
changes inside one launch, with hand-offs to the FP64 phase, and with
instances stopped by the iteration cap."""
import numpy as np
import pytest

from co_cultivation_metabolic_atlas_b200 import synthetic as syn
from oracle import dfba
from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="CUDA device required")]


def solve(models, species, lower, upper, cost, pair, config=None, warm=None):
    import torch
    from co_cultivation_metabolic_atlas_b200.engine import EngineOptions, LPEngine, SolveConfig
    eng = LPEngine([(m.S, m.S.shape[0]) for m in models], options=EngineOptions(pair_instances=pair))
    eng.set_instances(species, lower, upper, cost)
    kw = {} if warm is None else dict(warm_x=warm[0], warm_y=warm[1], warm_omega=warm[2])
    res = eng.solve(config=config or SolveConfig(), **kw)
    torch.cuda.synchronize()
    kinds = eng.phase_kernels()
    out = {k: getattr(res, k).cpu().numpy() for k in ("status", "objective", "x", "y", "iterations", "metrics",
                                                      "omega")}
    eng.close()
    return out, kinds


def community_batch(envs, seed=0, models=None):
    models = models or syn.community_models()
    medium, biomass = syn.initial_environments(envs, seed=seed)
    species = np.repeat(np.arange(3, dtype=np.int32), envs)
    lower = np.concatenate([dfba.uptake_lower_bounds(m, medium, biomass, 0.05).ravel() for m in models])
    upper = np.concatenate([np.tile(m.upper, envs) for m in models])
    cost = np.concatenate([np.tile(m.cost, envs) for m in models])
    return models, species, lower, upper, cost


def assert_same(a, b):
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_pair_kernel_equals_single_kernel_on_a_community_batch():
    models, species, lower, upper, cost = community_batch(512)
    single, ks = solve(models, species, lower, upper, cost, pair=False)
    paired, kp = solve(models, species, lower, upper, cost, pair=True)
    assert ks[0] == "pdhg_recentred<staged>" and kp[0] == "pdhg_recentred_pair"
    assert (paired["status"] == 0).all()
    assert_same(single, paired)


def test_pair_kernel_equals_single_kernel_warm_started():
    """Warm starts from a perturbed previous solution (different iteration
    counts per instance, so slots refill at different times)."""
    models, species, lower, upper, cost = community_batch(400, seed=3)
    base, _ = solve(models, species, lower, upper, cost, pair=True)
    rng = np.random.default_rng(4)
    lower2 = lower * rng.uniform(0.9, 1.1, lower.shape)
    warm = (base["x"], base["y"], base["omega"])
    single, _ = solve(models, species, lower2, upper, cost, pair=False, warm=warm)
    paired, kp = solve(models, species, lower2, upper, cost, pair=True, warm=warm)
    assert kp[0] == "pdhg_recentred_pair"
    assert np.ptp(paired["iterations"]) > 0
    assert_same(single, paired)


def test_pair_kernel_equals_single_kernel_with_handoffs_and_the_cap():
    """A one-test stall rule and a short test period hand instances to the
    FP64 phase; a low cap stops others; both kernels agree on all of it."""
    from co_cultivation_metabolic_atlas_b200.engine import SolveConfig
    model, lower, upper = syn.single_species_workload(320)
    species = np.zeros(320, np.int32)
    cost = np.tile(model.cost, 320)
    for config in (SolveConfig(fp64_stall_checks=1, check_every=16), SolveConfig(max_iterations=700)):
        single, _ = solve([model], species, lower.ravel(), upper.ravel(), cost, pair=False, config=config)
        paired, kp = solve([model], species, lower.ravel(), upper.ravel(), cost, pair=True, config=config)
        assert kp[0] == "pdhg_recentred_pair"
        assert_same(single, paired)


def test_pair_kernel_fixed_iterations_equal_single_kernel():
    """A fixed number of iterations with restarts (no termination)."""
    from co_cultivation_metabolic_atlas_b200.engine import SolveConfig
    model, lower, upper = syn.binding_species_workload(300, m=300, n=900, seed=3)
    config = SolveConfig(max_iterations=640, tol_primal=0.0, tol_dual=0.0, tol_gap=0.0, fp64_stall_checks=0)
    species = np.zeros(300, np.int32)
    cost = np.tile(model.cost, 300)
    single, _ = solve([model], species, lower.ravel(), upper.ravel(), cost, pair=False, config=config)
    paired, kp = solve([model], species, lower.ravel(), upper.ravel(), cost, pair=True, config=config)
    assert kp[0] == "pdhg_recentred_pair" and (paired["iterations"] == 640).all()
    assert_same(single, paired)


def test_small_batches_keep_one_instance_per_cta():
    """Below two instances per CTA of a full grid the single-instance kernel
    keeps more SMs busy and is used."""
    models, species, lower, upper, cost = community_batch(8)
    _, kp = solve(models, species, lower, upper, cost, pair=True)
    assert kp[0] == "pdhg_recentred<staged>"
