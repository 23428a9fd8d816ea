"""48 h dFBA trajectory parity: the device-resident community loop against
the CPU oracle (fixture made by ``tests/golden/make_trajectory.py``: the
engine's algorithm and warm-start policy restated in NumPy, objectives pinned
to HiGHS at sampled steps).

What the LPs determine is pinned over all 960 steps: every LP's optimal
value (1e-6 relative), hence growth and the biomass trajectory (1e-4
relative); the device's coupling (uptake bounds from the state, Euler
updates from the fluxes) is checked step by step against the oracle's
restatement applied to the device's own state and fluxes.  The exchange
fluxes themselves are not determined by these LPs (each medium exchange flux
spans its whole bound range on the optimal face; see
``tests/test_oracle_pins.py``), so the metabolite trajectory of any two
solvers drifts apart; its deviation from the oracle is reported, not
asserted."""
import numpy as np
import pytest

from co_cultivation_metabolic_atlas_b200 import synthetic as syn
from oracle import dfba
from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="CUDA device required")]

REL = 1e-4  # trajectory tolerance (relative)


def test_48h_trajectory_matches_oracle(golden_dir):
    import torch
    from co_cultivation_metabolic_atlas_b200.dfba import DeviceCommunity
    g = np.load(golden_dir / "trajectory_community.npz")
    envs = int(g["envs"])
    dt = float(g["dt"])
    steps = g["objective"].shape[0]
    kept = {int(k) for k in g["steps"]}
    models = syn.community_models(seed=0)
    medium, biomass = syn.initial_environments(envs, seed=int(g["seed"]))
    com = DeviceCommunity(models, medium, biomass, dt=dt, warm_start="extrapolate")
    n = [m.S.shape[1] for m in models]
    co = com.col_offsets.cpu().numpy()
    med, bio, obj = [], [], []
    coupling_err = bounds_err = 0.0
    for k in range(steps):
        m0 = com.medium.cpu().numpy()
        b0 = com.biomass.cpu().numpy()
        if k in kept:
            med.append(m0)
            bio.append(b0)
        com.uptake_bounds()
        lower = com.lower.cpu().numpy()
        for s, mdl in enumerate(models):
            ref_lo = dfba.uptake_lower_bounds(mdl, m0, b0, dt)
            got = lower[co[s * envs]:co[s * envs] + envs * n[s]].reshape(envs, n[s])
            bounds_err = max(bounds_err, float(np.abs(got - ref_lo).max()))
        res = com.solve()
        assert int(com.certified(res).item()) == envs * 3
        com.integrate(res)
        x = res.x.cpu().numpy()
        fluxes = [x[co[s * envs]:co[s * envs] + envs * n[s]].reshape(envs, n[s]) for s in range(3)]
        mu = np.stack([fluxes[s][:, models[s].biomass] for s in range(3)], axis=1)
        nb = dfba.update_biomass(b0, mu, dt)
        nm = dfba.update_medium(m0, models, fluxes, b0, dt)
        coupling_err = max(coupling_err,
                           float(np.abs(com.biomass.cpu().numpy() - nb).max() / max(1.0, np.abs(nb).max())),
                           float(np.abs(com.medium.cpu().numpy() - nm).max() / max(1.0, np.abs(nm).max())))
        obj.append(res.objective.view(3, envs).t().cpu().numpy())
    torch.cuda.synchronize()
    com.close()
    assert bounds_err <= 1e-12
    assert coupling_err <= 1e-12
    obj = np.stack(obj)
    ref_obj = g["objective"]
    assert np.all(np.abs(obj - ref_obj) <= 1e-6 * np.maximum(1.0, np.abs(ref_obj)))
    bio, med = np.stack(bio), np.stack(med)
    rb, rm = g["biomass"], g["medium"]
    err_b = np.abs(bio - rb) / np.maximum(np.abs(rb), 1e-12)
    err_m = np.abs(med - rm) / np.maximum(np.abs(rm), 1e-3 * np.abs(rm[0]).max())
    print(f"48 h trajectory vs oracle: max rel biomass error {err_b.max():.2e}; metabolites (not determined "
          f"by the LPs) max rel deviation {err_m.max():.2e} at 48 h, {err_m[:2].max():.2e} after 0.5 h")
    assert err_b.max() <= REL


# --- the parsimonious second stage: a unique optimum, so metabolites pin ---

def parsimonious_community(envs, seed):
    from co_cultivation_metabolic_atlas_b200.dfba import DeviceCommunity
    models = syn.community_models(seed=syn.BINDING_SEED, conserved=True)
    medium, biomass = syn.initial_environments(envs, seed=seed)
    return models, DeviceCommunity(models, medium, biomass, warm_start="extrapolate", parsimonious=True)


def test_parsimonious_stage_matches_highs_fluxes():
    """One step of the weight-conserving community: every stage-2 LP is
    certified, its objective equals HiGHS's, and so do its exchange fluxes
    (the weighted tie-break has a unique optimum)."""
    import torch
    from co_cultivation_metabolic_atlas_b200.parsimonious import exchange_weights
    envs = 6
    models, com = parsimonious_community(envs, seed=1)
    com.uptake_bounds()
    lower = com.lower.cpu().numpy()
    res = com.solve()
    res2 = com.solve_stage2(res)
    torch.cuda.synchronize()
    assert int(com.certified(res).item()) == envs * 3 and int(com.certified(res2).item()) == envs * 3
    x1 = res.x.cpu().numpy()
    v2 = com.stage2_fluxes(res2).cpu().numpy()
    obj2 = res2.objective.cpu().numpy()
    co = com.col_offsets.cpu().numpy()
    com.close()
    for s, m in enumerate(models):
        n = m.S.shape[1]
        for e in range(envs):
            i = s * envs + e
            lo = lower[co[i]:co[i] + n]
            status, v = dfba.parsimonious_fluxes(m, s, lo, m.upper, float(x1[co[i] + m.biomass]))
            assert status == 0
            got = v2[co[i]:co[i] + n]
            w = exchange_weights(m, s)
            ref_obj = float(w @ np.abs(v[:m.n_exchange]))
            assert abs(obj2[i] - ref_obj) <= 1e-6 * max(1.0, abs(ref_obj))
            scale = max(1.0, np.abs(v[:m.n_exchange]).max())
            assert np.abs(got[:m.n_exchange] - v[:m.n_exchange]).max() <= 1e-5 * scale


def test_parsimonious_48h_trajectory_matches_highs_oracle(golden_dir):
    """48 h (960 steps) of 4 environments with the parsimonious second
    stage against the trajectory of the same dFBA solved by HiGHS
    (``tests/golden/make_parsimonious_trajectory.py``): biomass AND medium
    within 1e-4 relative (max norm per step) over every step."""
    import torch
    path = golden_dir / "trajectory_parsimonious.npz"
    if not path.exists():
        pytest.skip("fixture not generated")
    g = np.load(path)
    envs, steps = int(g["envs"]), int(g["steps"])
    models, com = parsimonious_community(envs, seed=0)
    err_b = err_m = 0.0
    cert = 0
    for k in range(steps):
        st = com.step()
        cert += int(st.certified.item())
        rb, rm = g["biomass"][k + 1], g["medium"][k + 1]
        err_b = max(err_b, float(np.abs(com.biomass.cpu().numpy() - rb).max() / np.abs(rb).max()))
        err_m = max(err_m, float(np.abs(com.medium.cpu().numpy() - rm).max() / np.abs(rm).max()))
    torch.cuda.synchronize()
    com.close()
    print(f"parsimonious 48 h trajectory vs HiGHS: max rel biomass error {err_b:.2e}, medium {err_m:.2e}")
    assert cert == steps * envs * 3 * 2
    assert err_b <= REL and err_m <= REL
