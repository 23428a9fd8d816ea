"""Generate the 48 h dFBA trajectory fixture (``trajectory_community.npz``).

The oracle rolls a few environments of the seeded three-species community
forward for 960 explicit-Euler steps (dt = 0.05 h) on the CPU, with the
engine's algorithm restated in NumPy (``oracle.pdhg.solve_mixed``: re-centred
FP32 phase, FP64 hand-off, cold fallback) and the engine's warm-start policy
(step 0 cold, step 1 the previous solution, later steps the extrapolation of
the last two), and the dFBA coupling of ``oracle.dfba`` (uptake bounds,
biomass and medium updates).  Every 10th state (and the last) is stored.
HiGHS objectives of the LPs of a few sampled steps are stored beside the
oracle's, so the fixture itself is pinned to HiGHS.

The medium trajectory depends on which optimal fluxes the solver returns
(the LPs' optimal faces are not single points), so it is reproducible only
by the same algorithm with the same warm starts; HiGHS pins the objectives.

Usage:  python tests/golden/make_trajectory.py [--envs 4] [--steps 960] [--workers 4]
"""

from __future__ import annotations

import argparse
import multiprocessing as mp
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

SEED = 11          # environments (disjoint from the bench and training seeds)
DT = 0.05
EVERY = 10
HIGHS_STEPS = (0, 120, 480, 959)
# the fixture was generated with the primal-weight smoothing 0.5 (the
# engine's default); the rollout pins it so that re-running the first steps
# reproduces the fixture bit for bit whatever the default becomes
FIXTURE_OMEGA_SMOOTHING = 0.5


def rollout(env, envs, steps):
    """``_rollout`` with the fixture's primal-weight smoothing (restored
    afterwards)."""
    from oracle import pdhg
    old = pdhg.OMEGA_SMOOTHING
    pdhg.OMEGA_SMOOTHING = FIXTURE_OMEGA_SMOOTHING
    try:
        return _rollout(env, envs, steps)
    finally:
        pdhg.OMEGA_SMOOTHING = old


def _rollout(env, envs, steps):
    from co_cultivation_metabolic_atlas_b200 import synthetic as syn
    from oracle import dfba, pdhg
    models = syn.community_models(seed=0)
    medium_all, biomass_all = syn.initial_environments(envs, seed=SEED)
    medium = medium_all[env:env + 1].copy()
    biomass = biomass_all[env:env + 1].copy()
    prep = [pdhg.prepare(m.S) for m in models]
    hist = [[] for _ in models]          # per species: last two (x, y, omega)
    states = {"medium": [], "biomass": [], "objective": [], "iterations": [], "lower": {}}
    for k in range(steps):
        if k % EVERY == 0 or k == steps - 1:
            states["medium"].append((k, medium[0].copy()))
            states["biomass"].append((k, biomass[0].copy()))
        objs, its = [], []

        def solve(s, lower):
            mdl = models[s]
            h = hist[s]
            if not h:
                kw = {}
            elif len(h) == 1:
                kw = dict(x0=h[-1][0], y0=h[-1][1], omega0=h[-1][2])
            else:
                kw = dict(x0=2 * h[-1][0] - h[-2][0], y0=2 * h[-1][1] - h[-2][1], omega0=h[-1][2])
            r = pdhg.solve_mixed(prep[s], lower[0], mdl.upper, mdl.cost, **kw)
            h.append((r["x"], r["y"], r["omega"]))
            del h[:-2]
            objs.append(r["metrics"]["objective"])
            its.append(r["iterations"])
            if k in HIGHS_STEPS:
                states["lower"][(k, s)] = lower[0].copy()
            return (np.array([r["status"]]), np.array([r["x"][mdl.biomass]]), r["x"][None, :])

        medium, biomass, _ = dfba.step(models, medium, biomass, DT, solve)
        states["objective"].append(objs)
        states["iterations"].append(its)
    return env, states


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--envs", type=int, default=4)
    ap.add_argument("--steps", type=int, default=960)
    ap.add_argument("--workers", type=int, default=4)
    args = ap.parse_args()
    t0 = time.time()
    ctx = mp.get_context("spawn")
    with ctx.Pool(args.workers) as pool:
        res = pool.starmap(rollout, [(e, args.envs, args.steps) for e in range(args.envs)])
    res.sort(key=lambda r: r[0])
    from co_cultivation_metabolic_atlas_b200 import synthetic as syn
    from oracle import highs
    models = syn.community_models(seed=0)
    steps_kept = np.array([k for k, _ in res[0][1]["medium"]])
    medium = np.stack([[m for _, m in r[1]["medium"]] for r in res], axis=1)     # (K, E, 40)
    biomass = np.stack([[b for _, b in r[1]["biomass"]] for r in res], axis=1)   # (K, E, 3)
    objective = np.stack([np.array(r[1]["objective"]) for r in res], axis=1)     # (steps, E, 3)
    iterations = np.stack([np.array(r[1]["iterations"]) for r in res], axis=1)
    hs = np.array([k for k in HIGHS_STEPS if k < args.steps])
    highs_obj = np.full((len(hs), args.envs, len(models)), np.nan)
    for a, k in enumerate(hs):
        for e, r in enumerate(res):
            for s, mdl in enumerate(models):
                st, fun, _, _ = highs.solve_one(mdl.S, r[1]["lower"][(int(k), s)], mdl.upper, mdl.cost)
                if st == 0:
                    highs_obj[a, e, s] = fun
    np.savez_compressed(HERE / "trajectory_community.npz", steps=steps_kept, medium=medium, biomass=biomass,
                        objective=objective, iterations=iterations, highs_steps=hs, highs_objective=highs_obj,
                        seed=SEED, dt=DT, envs=args.envs)
    print(f"wrote trajectory_community.npz: {args.envs} envs x {args.steps} steps in {time.time() - t0:.0f} s; "
          f"mean iterations {iterations.mean():.1f}")


if __name__ == "__main__":
    main()
