"""The multi-GPU path's host logic on two CPU ranks (gloo): every rank gets
its own environments, training seeds never collide with any rank's
evaluation environments, and the job's rate is the sum of the ranks' units
over the slowest rank's time."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    from co_cultivation_metabolic_atlas_b200 import synthetic as syn
    from co_cultivation_metabolic_atlas_b200.distributed import Ranks, job_rate
    from oracle import dfba
    ranks = Ranks("gloo", timeout_s=60)
    medium, biomass = syn.initial_environments(16, seed=ranks.environment_seed(0))
    models = syn.community_models()
    lowers = [dfba.uptake_lower_bounds(m, medium, biomass, 0.05) for m in models]
    units = float(sum(len(lw) for lw in lowers))
    seconds = 0.5 + rank                      # a stand-in for a measured device time
    envs = [None] * world
    dist.all_gather_object(envs, medium.tobytes())
    seeds = [None] * world
    dist.all_gather_object(seeds, (ranks.environment_seed(0), ranks.training_seeds(0, 2)))
    rate = job_rate(units, seconds, ranks)
    ranks.barrier()
    if rank == 0:
        out.put(dict(envs=envs, seeds=seeds, rate=rate, units=units))
    ranks.close()


def test_two_cpu_ranks_shard_environments_and_reduce_scalars():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = out.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res["envs"][0] != res["envs"][1]                 # disjoint environment sets
    eval_seeds = {s for s, _ in res["seeds"]}
    train_seeds = {t for _, ts in res["seeds"] for t in ts}
    assert not eval_seeds & train_seeds
    assert res["rate"] == pytest.approx(2 * res["units"] / 1.5)  # sum of units / slowest rank
