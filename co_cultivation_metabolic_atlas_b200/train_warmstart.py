"""Train the learned warm start on the engine's own dFBA rollouts.

    python -m co_cultivation_metabolic_atlas_b200.train_warmstart --out PATH
        [--envs 4096] [--steps 48] [--seeds 1 2 ...] [--epochs 20]

Data: for each training seed, ``--envs`` environments are rolled forward
``--steps`` dFBA steps with extrapolated warm starts; every certified
(environment, step) contributes one (state features -> concatenated x, y of
the three species) pair.  The seeds must differ from the evaluation seeds.
The artifact holds the network weights, the codec, the architecture and a
hash of the species matrices it was trained for.
"""

from __future__ import annotations

import argparse
import hashlib
import time

import numpy as np
import torch

from . import synthetic as syn
from .engine import SolveConfig
from .warmstart import MLP, Codec, LearnedWarmStart, Rollouts, collect, train

HIDDEN = (512, 512, 512, 512)
N_FEATURES = 44


def models_digest(models):
    h = hashlib.sha256()
    for m in models:
        for a in (m.S.data, m.S.indices, m.S.indptr, m.lower, m.upper, m.cost, m.medium_columns, m.medium_ids,
                  m.vmax, m.km):
            h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def build_dataset(models, *, envs, steps, seeds, config=None, device=None, log=print) -> Rollouts:
    parts = []
    for sd in seeds:
        t0 = time.perf_counter()
        r = collect(models, envs=envs, steps=steps, seed=sd, config=config, device=device)
        ok = r.ok
        parts.append(Rollouts(r.F[ok], r.T[ok], ok[ok], r.omega[ok]))
        log(f"seed {sd}: {int(ok.sum())}/{len(ok)} certified pairs in {time.perf_counter() - t0:.1f} s")
    return Rollouts(*(torch.cat([getattr(p, f) for p in parts]) for f in ("F", "T", "ok", "omega")))


def fit(models, data: Rollouts, *, epochs=20, batch=4096, lr=1e-3, lr_final=5e-5, seed=0, device=None,
        log=print, ranks=None):
    """Train the network (state -> solution) on standardised targets;
    returns the warm start and the per-epoch losses.  With ``ranks`` of a
    multi-GPU job the training is data-parallel over every rank's rollouts
    (global standardisation, gradients averaged each step; the same
    network on every rank)."""
    from .distributed import min_int
    omega = data.omega.median(dim=0).values
    codec = Codec.fit(data.F, data.T, omega, ranks=ranks)
    width = data.T.shape[1]
    net = MLP([N_FEATURES, *HIDDEN, width], device=device, seed=seed)
    losses = train(net, codec.features(data.F), codec.targets(data.T), epochs=epochs,
                   batch=min_int(min(batch, data.F.shape[0]), ranks), lr=lr, lr_final=lr_final, seed=seed,
                   log=log, ranks=ranks)
    return LearnedWarmStart(net, codec, models), losses


def save(path, ws: LearnedWarmStart, models, meta):
    torch.save({"mlp": ws.mlp.state_dict(), "codec": ws.codec.state_dict(), "digest": models_digest(models),
                "meta": meta}, path)


def load(path, models, device=None):
    blob = torch.load(path, map_location="cpu", weights_only=True)
    if blob["digest"] != models_digest(models):
        raise ValueError("warm-start artifact was trained for different species matrices")
    dev = torch.device(device) if device is not None else torch.device("cuda")
    sd = blob["mlp"]
    net = MLP(sd["dims"], device=dev)
    net.load_state_dict(sd)
    codec = Codec.from_state(blob["codec"], dev)
    return LearnedWarmStart(net, codec, models), blob.get("meta", {})


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--envs", type=int, default=4096)
    ap.add_argument("--steps", type=int, default=48)
    ap.add_argument("--seeds", type=int, nargs="+", default=[101, 102])
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--model-seed", type=int, default=0)
    args = ap.parse_args()
    models = syn.community_models(seed=args.model_seed)
    data = build_dataset(models, envs=args.envs, steps=args.steps, seeds=args.seeds, config=SolveConfig())
    ws, losses = fit(models, data, epochs=args.epochs)
    save(args.out, ws, models, {"pairs": int(data.F.shape[0]), "losses": losses, "seeds": args.seeds})
    print(f"saved {args.out}: {data.F.shape[0]} pairs, final mse {losses[-1]:.4e}")


if __name__ == "__main__":
    main()
