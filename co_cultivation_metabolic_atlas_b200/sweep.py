"""Scale and degeneracy sweep: three large species (3,000 x 6,000,
2,500 x 5,200, 3,400 x 6,800; fixed exchange bounds, duplicated reversible
columns), uneven batches of 1k / 4k / 16k / 64k instances in one launch.

    python -m co_cultivation_metabolic_atlas_b200.sweep [--batches 1024 4096 16384 65536]
        [--autotune] [--cache PATH]

For every batch size: a cold solve of the whole batch, then a warm-started
re-solve after a perturbation of every free exchange bound (the previous
solutions as seeds, as in a dFBA step), and with ``--learned`` the same
cold batch seeded by the learned warm start (one request network per
species -- ``warmstart.RequestWarmStart``'s members -- trained on cold
solves of training batches drawn with other seeds).  Prints one JSON line
per batch: certified LPs/s, iteration distribution, streaming-model GB/s of
the re-centred phase and the launch configuration (autotuned per batch with
``--autotune``).
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import synthetic as syn
from .engine import EngineOptions, LPEngine, SolveConfig


def device_batch(models, count, mix, seed, device):
    """Flat device arrays of an uneven scale batch (species-major)."""
    sid, bounds = None, []
    gen = torch.Generator(device=device).manual_seed(seed)
    sizes = np.floor(np.asarray(mix, float) / np.sum(mix) * count).astype(int)
    sizes[0] += count - sizes.sum()
    sid = np.repeat(np.arange(len(models), dtype=np.int32), sizes)
    lows, ups, costs, free_idx = [], [], [], []
    for s, mdl in enumerate(models):
        k = int(sizes[s])
        lo = torch.as_tensor(mdl.lower, device=device).repeat(k, 1)
        free = np.flatnonzero(mdl.lower[:mdl.n_exchange] < mdl.upper[:mdl.n_exchange])
        draw = -20.0 * torch.rand((k, len(free)), generator=gen, device=device, dtype=torch.float64)
        if mdl.anchor is not None:
            draw = torch.minimum(draw, torch.as_tensor(mdl.anchor[free], device=device)[None, :])
        lo[:, torch.as_tensor(free, device=device)] = draw
        lows.append(lo.reshape(-1))
        ups.append(torch.as_tensor(mdl.upper, device=device).repeat(k))
        costs.append(torch.as_tensor(mdl.cost, device=device).repeat(k))
        free_idx.append((k, free))
    return sid, torch.cat(lows), torch.cat(ups), torch.cat(costs), free_idx


def perturb(models, lower, free_idx, seed, device):
    """Scale every free exchange lower bound by U[0.95, 1.05] (anchors kept)."""
    gen = torch.Generator(device=device).manual_seed(seed)
    out = lower.clone()
    base = 0
    for mdl, (k, free) in zip(models, free_idx):
        n = mdl.S.shape[1]
        view = out[base:base + k * n].view(k, n)
        f = torch.as_tensor(free, device=device)
        scaled = view[:, f] * (0.95 + 0.1 * torch.rand((k, len(free)), generator=gen, device=device,
                                                       dtype=torch.float64))
        if mdl.anchor is not None:
            scaled = torch.minimum(scaled, torch.as_tensor(mdl.anchor[free], device=device)[None, :])
        view[:, f] = scaled
        base += k * n
    return out


def streaming_bytes(models, sid, iters):
    """Streaming-model bytes of the re-centred phase (w = 4)."""
    per = np.array([4 * (3 * m.S.shape[1] + 3 * m.S.shape[0] + 2 * len(m.medium_columns)) for m in models], float)
    inst = float(np.sum(iters * per[sid]))
    mat = 0.0
    for s, m in enumerate(models):
        its = iters[sid == s]
        mat += float(its.max() if its.size else 0) * 2 * (m.S.nnz * 8 + 4 * (m.S.shape[0] + 1))
    return inst + mat


def train_members(models, args, device, count=2048, seeds=(101, 102), epochs=20):
    """One request network per species, trained on cold solves of
    ``count``-instance training batches (seeds disjoint from the
    evaluation batches')."""
    from .warmstart import fit_request_member
    mats = [(m.S, m.S.shape[0]) for m in models]
    rows = [dict(lower=[], x=[], y=[], omega=[]) for _ in models]
    for sd in seeds:
        sid, lo, up, cost, _ = device_batch(models, count, args.mix, sd, device)
        eng = LPEngine(mats, device=device)
        eng.set_instances(sid, lo, up, cost)
        res = eng.solve(config=SolveConfig())
        co, ro, _, _ = eng.layout(sid)
        ok = (res.status == 0).cpu().numpy()
        lo_h, x_h, y_h, om = lo.cpu().numpy(), res.x.cpu().numpy(), res.y.cpu().numpy(), res.omega.cpu().numpy()
        for i in np.flatnonzero(ok):
            s, (m, n) = int(sid[i]), models[int(sid[i])].S.shape
            rows[s]["lower"].append(lo_h[co[i]:co[i] + n])
            rows[s]["x"].append(x_h[co[i]:co[i] + n])
            rows[s]["y"].append(y_h[ro[i]:ro[i] + m])
            rows[s]["omega"].append(om[i])
        eng.close()
    members = []
    for s, mdl in enumerate(models):
        d = {k: np.asarray(v) for k, v in rows[s].items()}
        k = d["lower"].shape[0]
        n, m = mdl.S.shape[1], mdl.S.shape[0]
        member, _ = fit_request_member(d["lower"], np.broadcast_to(mdl.upper, (k, n)),
                                       np.broadcast_to(mdl.cost, (k, n)), np.zeros((k, m)), d["x"], d["y"],
                                       d["omega"], epochs=epochs, device=device)
        members.append(member)
    return members


def learned_seed(models, members, sid, lower, eng, device):
    """Flat (x, y, omega) warm start of a batch from the species' networks."""
    co, ro, tc, tr = eng.layout(sid)
    wx = torch.zeros(tc, dtype=torch.float64, device=device)
    wy = torch.zeros(max(1, tr), dtype=torch.float64, device=device)
    wo = torch.ones(len(sid), dtype=torch.float64, device=device)
    lo_h = lower.cpu().numpy()
    for s, (mdl, mem) in enumerate(zip(models, members)):
        idx = np.flatnonzero(sid == s)
        if idx.size == 0:
            continue
        m, n = mdl.S.shape
        lo = np.stack([lo_h[co[i]:co[i] + n] for i in idx])
        k = len(idx)
        pred = mem.predict(mem.features(lo, np.broadcast_to(mdl.upper, (k, n)), np.broadcast_to(mdl.cost, (k, n)),
                                        np.zeros((k, m))))
        cols = torch.as_tensor(np.concatenate([co[i] + np.arange(n) for i in idx]), device=device)
        rows = torch.as_tensor(np.concatenate([ro[i] + np.arange(m) for i in idx]), device=device)
        wx[cols] = pred[:, :n].reshape(-1)
        wy[rows] = pred[:, n:].reshape(-1)
        wo[torch.as_tensor(idx, device=device)] = mem.omega
    return wx, wy[:tr], wo


def run(batch, models, args, device, members=None):
    sid, lo, up, cost, free_idx = device_batch(models, batch, args.mix, args.seed, device)
    mats = [(m.S, m.S.shape[0]) for m in models]
    opt, cfg, tuning = EngineOptions(), SolveConfig(), None
    eng0 = LPEngine(mats, options=opt, device=device)
    eng0.set_instances(sid, lo, up, cost)
    co = eng0.col_offsets
    if args.autotune:
        from .autotune import autotune
        opt, cfg, tuning = autotune(mats, sid, lo, up, cost, co, cache=args.cache, device=device)
        eng0.close()
        eng0 = LPEngine(mats, options=opt, device=device)
        eng0.set_instances(sid, lo, up, cost)
    eng = eng0
    out = {"batch": batch, "mix": list(args.mix), "warps_per_block": opt.warps_per_block,
           "check_every": cfg.check_every}
    results = {}
    phases = ("cold", "learned", "warm") if members is not None else ("cold", "warm")
    for phase in phases:
        kw = {}
        if phase == "learned":
            wx, wy, wo = learned_seed(models, members, sid, lo, eng, device)
            kw = dict(warm_x=wx, warm_y=wy, warm_omega=wo)
        if phase == "warm":
            prev = results["cold_res"]
            lo2 = perturb(models, lo, free_idx, args.seed + 1, device)
            eng.set_instances(sid, lo2, up, cost)
            kw = dict(warm_x=prev.x[:eng.total_cols], warm_y=prev.y[:eng.total_rows], warm_omega=prev.omega)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record()
        res = eng.solve(config=cfg, **kw)
        stop.record()
        torch.cuda.synchronize()
        ms = start.elapsed_time(stop)
        t32, t64 = eng.phase_times()
        it = res.iterations.cpu().numpy().astype(np.int64)
        st = res.status.cpu().numpy()
        mt = res.metrics.cpu().numpy()
        cert = int(np.sum((st == 0) & (mt[:, 0] <= 1e-5) & (mt[:, 1] <= 1e-7) & (mt[:, 2] <= 1e-7)))
        it32 = eng.phase_iterations().cpu().numpy().astype(np.int64)
        gbs = streaming_bytes(models, sid, it32) / (t32 / 1e3) / 1e9 if t32 > 0 else None
        device_ms = t32 + t64  # the two phase launches (the call's wall time also holds first-call set-up)
        out[phase] = {"ms": ms, "device_ms": device_ms, "certified": cert, "lps_per_s": cert / (device_ms / 1e3),
                      "iterations": {"mean": float(it.mean()), "p50": float(np.median(it)),
                                     "p90": float(np.percentile(it, 90)), "p99": float(np.percentile(it, 99)),
                                     "max": int(it.max())},
                      "fp64_handoffs": int(np.sum(it > it32)), "first_phase_ms": t32, "fp64_phase_ms": t64,
                      "streaming_model_gbs": gbs}
        results[phase + "_res"] = res
    if tuning is not None:
        out["autotune"] = tuning
    eng.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--batches", type=int, nargs="+", default=[1024, 4096, 16384, 65536])
    ap.add_argument("--mix", type=float, nargs=3, default=[0.5, 0.3, 0.2])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--cache", default=None)
    ap.add_argument("--learned", action="store_true",
                    help="also solve each cold batch from the learned warm start (networks trained first)")
    args = ap.parse_args()
    device = torch.device("cuda", 0)
    t0 = time.perf_counter()
    models = syn.community_models(syn.LARGE_SIZES, fixed_fraction=0.2, duplicate_fraction=0.05)
    print(json.dumps({"workload": "scale sweep: species " + ", ".join(f"{m.S.shape[0]}x{m.S.shape[1]}" for m in models),
                      "generator_seconds": time.perf_counter() - t0}), flush=True)
    members = None
    if args.learned:
        t1 = time.perf_counter()
        members = train_members(models, args, device)
        print(json.dumps({"learned_training_seconds": time.perf_counter() - t1}), flush=True)
    for b in args.batches:
        print(json.dumps(run(b, models, args, device, members)), flush=True)


if __name__ == "__main__":
    main()
