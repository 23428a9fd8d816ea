"""Autotuner for the batched LP engine.

The engine's launch shape and test period are tunable: instances per CTA in
the re-centred phase (1, or 2 sharing one staged matrix: the width of the
sparse-matrix times dense-block tile), warps per block (the SELL-32 slice
schedule, one lane per row, is rebalanced per warp count, which sets the
rows each warp walks per pass), and ``check_every``, the period of the FP64
convergence tests at which restarts are decided.  ``autotune`` times a seeded sample of the batch
(every species represented, solved to the production tolerances) for every
candidate and keeps the fastest per certified LP; results are cached in a
JSON file keyed by the species matrices' shapes and nonzero counts and the
device name, so a later run of the same workload reuses the choice.
"""

from __future__ import annotations

import hashlib
import itertools
import json
import time
from dataclasses import replace
from pathlib import Path

import numpy as np
import torch

from .engine import EngineOptions, LPEngine, SolveConfig

WARPS = (8, 16, 32)
CHECK_EVERY = (32, 64, 128)
PAIR = (True, False)


def workload_key(matrices, device=None) -> str:
    h = hashlib.sha256()
    for a, neq in matrices:
        h.update(np.asarray([a.shape[0], a.shape[1], a.nnz, neq], dtype=np.int64).tobytes())
    name = torch.cuda.get_device_name(device) if torch.cuda.is_available() else "none"
    h.update(name.encode())
    return h.hexdigest()[:24]


def _sample(species_id, count):
    """Instance indices of a seeded sample with every species represented."""
    rng = np.random.default_rng(12345)
    sid = np.asarray(species_id)
    picks = []
    per = max(1, count // len(np.unique(sid)))
    for s in np.unique(sid):
        idx = np.flatnonzero(sid == s)
        picks.append(np.sort(rng.choice(idx, min(per, len(idx)), replace=False)))
    return np.concatenate(picks)


def autotune(matrices, species_id, lower, upper, cost, col_offsets, *, config: SolveConfig | None = None,
             sample=592, warps=WARPS, check_every=CHECK_EVERY, pair=PAIR, cache: str | Path | None = None,
             device=None, log=None):
    """Pick ``(EngineOptions, SolveConfig)`` for a batch.

    ``matrices``: the engine's ``(A, neq)`` list; ``species_id``: per
    instance; ``lower``/``upper``/``cost``: flat device tensors of the batch
    with instance ``i`` at ``col_offsets[i]``.  Returns the chosen options,
    config and the per-candidate timings.
    """
    config = config or SolveConfig()
    key = workload_key(matrices, device)
    if cache is not None and Path(cache).exists():
        table = json.loads(Path(cache).read_text())
        if key in table:
            best = table[key]
            return (replace(EngineOptions(), warps_per_block=best["warps_per_block"],
                            pair_instances=best.get("pair_instances", True)),
                    replace(config, check_every=best["check_every"]), best["timings"])
    pick = _sample(species_id, sample)
    sid = np.asarray(species_id)[pick].astype(np.int32)
    n = np.array([a.shape[1] for a, _ in matrices])
    cols = [torch.arange(int(col_offsets[i]), int(col_offsets[i]) + int(n[species_id[i]]), device=lower.device)
            for i in pick]
    cols = torch.cat(cols)
    lo, up, c = lower[cols].contiguous(), upper[cols].contiguous(), cost[cols].contiguous()
    timings = []
    for w, ce, pr in itertools.product(warps, check_every, pair):
        try:
            eng = LPEngine(matrices, options=replace(EngineOptions(), warps_per_block=w, pair_instances=pr),
                           device=device)
        except Exception as exc:  # a launch shape this device cannot run
            timings.append({"warps_per_block": w, "check_every": ce, "pair_instances": pr, "error": str(exc)})
            continue
        eng.set_instances(sid, lo, up, c)
        cfg = replace(config, check_every=ce)
        eng.solve(config=cfg)                      # warm-up (staging, layouts)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = eng.solve(config=cfg)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        ok = int((res.status == 0).sum().item())
        kernel = eng.phase_kernels()[0]
        eng.close()
        row = {"warps_per_block": w, "check_every": ce, "pair_instances": pr, "kernel": kernel, "seconds": dt,
               "certified": ok, "seconds_per_certified_lp": dt / max(ok, 1)}
        timings.append(row)
        if log:
            log(row)
    valid = [t for t in timings if "error" not in t and t["certified"] == len(pick)] or \
            [t for t in timings if "error" not in t]
    best = min(valid, key=lambda t: t["seconds_per_certified_lp"])
    if cache is not None:
        table = json.loads(Path(cache).read_text()) if Path(cache).exists() else {}
        table[key] = dict(best, timings=timings)
        tmp = Path(str(cache) + ".tmp")
        tmp.write_text(json.dumps(table, indent=1))
        tmp.replace(cache)
    return (replace(EngineOptions(), warps_per_block=best["warps_per_block"], pair_instances=best["pair_instances"]),
            replace(config, check_every=best["check_every"]), timings)
