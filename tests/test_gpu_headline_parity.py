"""Parity at the headline configuration, through the C ABI.

* One seeded 4,096-environment step of the three-species community (12,288
  LPs per step, mixed precision, learned warm start): every LP's in-kernel
  FP64 certificate (primal residual, dual violation, relative KKT gap)
  equals the oracle's certificate of the returned (x, y), and 512 LPs per
  species match HiGHS's objective to 1e-6 relative.
* The uptake-binding families (weight-conserving species), whose optimal
  values differ per instance: the single-species batch and a 1,024-environment
  community step, against HiGHS instance by instance.

Certificate tolerance: ``|kernel - oracle| <= 1e-9 |oracle| + floor``, with
``floor`` the FP64 evaluation-order bound of that quantity (64 eps times the
magnitude of the terms it sums: row l1 norm of |S| times |x|_inf for the
primal residual, |c|_inf plus column l1 norm times |y|_inf for the dual
violation, their product over the columns divided by max(1, |c.x|) for the
KKT gap).  The kernel evaluates in scaled space in another order, so the
values agree to rounding, not bit for bit.
"""
import numpy as np
import pytest

from co_cultivation_metabolic_atlas_b200 import synthetic as syn
from oracle import certificate, highs
from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="CUDA device required")]

ENVS = 4096
PER_SPECIES = 512
OBJ_TOL = 1e-6
EPS = np.finfo(np.float64).eps


def species_blocks(com, res, lower):
    """Per species: (model, X, Y, L, objective, metrics, status) of one step."""
    E = com.E
    x = res.x.cpu().numpy()
    y = res.y.cpu().numpy()
    obj = res.objective.cpu().numpy()
    mt = res.metrics.cpu().numpy()
    st = res.status.cpu().numpy()
    co, ro, _, _ = com.engine.layout(com.species_id)
    out = []
    for s, m in enumerate(com.models):
        rows, n = m.S.shape
        c0, r0 = int(co[s * E]), int(ro[s * E])
        sl = slice(s * E, (s + 1) * E)
        out.append((m, x[c0:c0 + E * n].reshape(E, n), y[r0:r0 + E * rows].reshape(E, rows),
                    lower[c0:c0 + E * n].reshape(E, n), obj[sl], mt[sl], st[sl]))
    return out


def assert_certificates_match(model, X, Y, L, metrics):
    """The kernel's metrics[:, 0:3] equal the oracle's certificate of (X, Y)."""
    S = model.S
    U = np.broadcast_to(model.upper, X.shape)
    p, d, g = certificate.certificate_rows(S, np.zeros(S.shape[0]), L, U, model.cost, S.shape[0], X, Y)
    absS = abs(S)
    row_l1 = float(np.asarray(absS.sum(axis=1)).max())
    col_l1 = float(np.asarray(absS.sum(axis=0)).max())
    xinf = np.abs(X).max(axis=1)
    yinf = np.abs(Y).max(axis=1)
    cinf = float(np.abs(model.cost).max())
    fl_p = 64 * EPS * row_l1 * np.maximum(1.0, xinf)
    fl_d = 64 * EPS * (cinf + col_l1 * np.maximum(1.0, yinf))
    fl_g = fl_d * np.maximum(1.0, xinf) * S.shape[1] / np.maximum(1.0, np.abs(X @ model.cost))
    for name, k, o, fl in (("primal", metrics[:, 0], p, fl_p), ("dual", metrics[:, 1], d, fl_d),
                           ("gap", metrics[:, 2], g, fl_g)):
        bad = np.abs(k - o) > 1e-9 * np.abs(o) + fl
        assert not bad.any(), (f"{name}: {int(bad.sum())} of {len(k)} differ; worst kernel "
                               f"{k[bad][:3]} oracle {o[bad][:3]}")


def highs_objectives(model, L, idx):
    res, _ = highs.solve_batch([model.S] * len(idx), [L[i] for i in idx], [model.upper] * len(idx),
                               [model.cost] * len(idx))
    assert all(r[0] == 0 for r in res)
    return np.array([r[1] for r in res])


@pytest.fixture(scope="module")
def headline_steps():
    """Steps 0 (the network's seed) and 2 (the temporal base) of a seeded
    4,096-environment learned-warm-start rollout, with the bounds each step
    was solved with."""
    import torch
    from co_cultivation_metabolic_atlas_b200 import train_warmstart as tw
    from co_cultivation_metabolic_atlas_b200.dfba import DeviceCommunity
    models = syn.community_models()
    data = tw.build_dataset(models, envs=1024, steps=8, seeds=[401, 402], log=lambda *_: None)
    ws, _ = tw.fit(models, data, epochs=4, batch=1024, log=lambda *_: None)
    medium, biomass = syn.initial_environments(ENVS, seed=0)
    com = DeviceCommunity(models, medium, biomass, warm_start="learned", learned=ws)
    steps = {}
    for k in range(3):
        com.uptake_bounds()
        lower = com.lower.cpu().numpy()
        res = com.solve()
        torch.cuda.synchronize()
        steps[k] = species_blocks(com, res, lower)
        com.integrate(res)
    com.close()
    return steps


@pytest.mark.parametrize("step", [0, 2])
def test_every_lp_of_a_headline_step_is_certified_and_its_certificate_matches_the_oracle(headline_steps, step):
    for model, X, Y, L, obj, mt, st in headline_steps[step]:
        assert (st == 0).all()
        assert (mt[:, 0] <= 1e-5).all() and (mt[:, 1] <= 1e-7).all() and (mt[:, 2] <= 1e-7).all()
        assert_certificates_match(model, X, Y, L, mt)


def test_headline_step_objectives_match_highs_on_512_lps_per_species(headline_steps):
    rng = np.random.default_rng(12)
    for model, X, Y, L, obj, mt, st in headline_steps[2]:
        idx = np.sort(rng.choice(ENVS, PER_SPECIES, replace=False))
        ref = highs_objectives(model, L, idx)
        err = np.abs(obj[idx] - ref) / np.maximum(1.0, np.abs(ref))
        assert err.max() <= OBJ_TOL, err.max()
        # the returned objective is c.x of the returned fluxes
        np.testing.assert_allclose(obj[idx], X[idx] @ model.cost, rtol=1e-12, atol=1e-12)


def test_network_seeded_step_objectives_match_highs(headline_steps):
    rng = np.random.default_rng(13)
    for model, X, Y, L, obj, mt, st in headline_steps[0]:
        idx = np.sort(rng.choice(ENVS, 64, replace=False))
        ref = highs_objectives(model, L, idx)
        assert (np.abs(obj[idx] - ref) / np.maximum(1.0, np.abs(ref))).max() <= OBJ_TOL


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_binding_single_species_batch_matches_highs_per_instance(precision):
    """Uptake binds: 64 instances with 64 different optimal values, each
    equal to HiGHS's."""
    from co_cultivation_metabolic_atlas_b200.engine import LPEngine, SolveConfig
    count = 64
    model, lower, upper = syn.binding_species_workload(count)
    eng = LPEngine([(model.S, model.S.shape[0])])
    eng.set_instances(np.zeros(count, np.int32), lower.ravel(), upper.ravel(), np.tile(model.cost, count))
    res = eng.solve(config=SolveConfig(precision=precision))
    st = res.status.cpu().numpy()
    obj = res.objective.cpu().numpy()
    n, m = model.S.shape[1], model.S.shape[0]
    X = res.x.cpu().numpy()[:count * n].reshape(count, n)
    Y = res.y.cpu().numpy()[:count * m].reshape(count, m)
    mt = res.metrics.cpu().numpy()
    eng.close()
    assert (st == 0).all()
    ref = highs_objectives(model, lower, np.arange(count))
    assert np.ptp(ref) > 1.0  # the optimal values differ per instance
    assert (np.abs(obj - ref) / np.maximum(1.0, np.abs(ref))).max() <= OBJ_TOL
    assert_certificates_match(model, X, Y, lower, mt)


def test_binding_community_step_matches_highs_per_environment():
    """A 1,024-environment step of the weight-conserving community: growth
    depends on the medium, so every environment has its own optimum."""
    import torch
    from co_cultivation_metabolic_atlas_b200.dfba import DeviceCommunity
    E = 1024
    models = syn.community_models(seed=syn.BINDING_SEED, conserved=True)
    medium, biomass = syn.initial_environments(E, seed=5)
    com = DeviceCommunity(models, medium, biomass, warm_start="extrapolate")
    blocks = None
    for _ in range(3):
        com.uptake_bounds()
        lower = com.lower.cpu().numpy()
        res = com.solve()
        torch.cuda.synchronize()
        blocks = species_blocks(com, res, lower)
        com.integrate(res)
    com.close()
    rng = np.random.default_rng(3)
    for model, X, Y, L, obj, mt, st in blocks:
        assert (st == 0).all()
        assert_certificates_match(model, X, Y, L, mt)
        idx = np.sort(rng.choice(E, 128, replace=False))
        ref = highs_objectives(model, L, idx)
        assert np.ptp(ref) > 1e-3 * np.abs(ref).max()
        assert (np.abs(obj[idx] - ref) / np.maximum(1.0, np.abs(ref))).max() <= OBJ_TOL
