"""The multi-GPU path's host logic on two CPU ranks (gloo): every rank gets
its own environments, training seeds never collide with any rank's
evaluation environments, and the job's rate is the sum of the ranks' units
over the slowest rank's time."""
import os
import socket

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


def _dp_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch
    from co_cultivation_metabolic_atlas_b200.distributed import Ranks, allreduce_mean_, global_moments, min_int
    ranks = Ranks("gloo", timeout_s=60)
    g = torch.Generator().manual_seed(0)
    X = torch.randn(64, 5, generator=g)
    y = X @ torch.arange(1.0, 6.0) + 0.1 * torch.randn(64, generator=g)
    shard = slice(32 * rank, 32 * (rank + 1))
    mean, std = global_moments(X[shard] * (1 + rank), ranks)
    w = torch.zeros(5, requires_grad=True)
    for _ in range(25):
        loss = ((X[shard] @ w - y[shard]) ** 2).mean()
        (gw,) = torch.autograd.grad(loss, w)
        allreduce_mean_([gw], ranks)
        with torch.no_grad():
            w -= 0.05 * gw
    steps = min_int(10 + 7 * rank, ranks)
    out.put((rank, w.detach().clone(), mean, std, steps))
    ranks.close()


def test_data_parallel_training_helpers_on_two_cpu_ranks():
    """Gradients averaged by one all-reduce keep the replicas identical and
    equal to full-batch training; the standardisation moments are those of
    every rank's rows; step counts agree on the smallest."""
    import torch
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dp_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict((r, rest) for r, *rest in (out.get(timeout=120) for _ in range(2)))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = torch.Generator().manual_seed(0)
    X = torch.randn(64, 5, generator=g)
    y = X @ torch.arange(1.0, 6.0) + 0.1 * torch.randn(64, generator=g)
    w = torch.zeros(5, requires_grad=True)
    for _ in range(25):
        loss = ((X @ w - y) ** 2).mean()
        (gw,) = torch.autograd.grad(loss, w)
        with torch.no_grad():
            w -= 0.05 * gw
    torch.testing.assert_close(got[0][0], got[1][0], rtol=0, atol=0)
    torch.testing.assert_close(got[0][0], w.detach(), rtol=1e-5, atol=1e-6)
    both = torch.cat([X[:32], 2 * X[32:]])
    torch.testing.assert_close(got[0][1], both.mean(0), rtol=1e-6, atol=1e-6)
    torch.testing.assert_close(got[1][2], both.std(0), rtol=1e-6, atol=1e-6)
    assert got[0][3] == got[1][3] == 10
