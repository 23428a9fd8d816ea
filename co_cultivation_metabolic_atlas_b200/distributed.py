"""One process per GPU: environment sharding and the scalar reductions of a
multi-GPU run.

Every LP instance is independent and the dFBA couples species only inside
one environment, so a multi-GPU run gives each rank its own environments
(weak scaling: a fixed number per GPU) and shares nothing on the data path.
The data path has no collective; reporting uses scalar reductions (the
maximum of the per-rank device times, the sum of the per-rank counts).  The
learned warm start can be trained data-parallel: every rank rolls out its
own training environments, the codec's standardisation uses the moments of
all ranks' data, and each Adam step applies the gradient averaged over the
ranks by one flattened all-reduce, so the replicas stay identical.
``torch.distributed`` carries all of it (NCCL on GPUs, gloo on the CPU).
"""

from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


class Ranks:
    """The calling process's place in a ``torchrun`` job (a single process
    when WORLD_SIZE is unset)."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 600.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.device = None
        if self.world > 1 and not dist.is_initialized():
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
        if backend == "nccl":
            torch.cuda.set_device(self.local_rank)
            self.device = torch.device("cuda", self.local_rank)
        else:
            self.device = torch.device("cpu")

    def environment_seed(self, base: int) -> int:
        """Seed of this rank's environments: disjoint environment sets."""
        return base + 1000 * self.rank

    def training_seeds(self, base: int, count: int) -> list[int]:
        """Seeds of this rank's warm-start training rollouts, disjoint from
        every rank's evaluation environments (``environment_seed``)."""
        return [base + 1000 * (self.world + 1) + 100 * self.rank + k for k in range(count)]

    def barrier(self):
        if self.world > 1:
            dist.barrier()

    def _reduce(self, value: float, op) -> float:
        if self.world == 1:
            return float(value)
        t = torch.tensor([float(value)], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, value: float) -> float:
        return self._reduce(value, dist.ReduceOp.MAX)

    def sum(self, value: float) -> float:
        return self._reduce(value, dist.ReduceOp.SUM)

    def close(self):
        if self.world > 1 and dist.is_initialized():
            dist.destroy_process_group()


def job_rate(units_per_rank: float, seconds_per_rank: float, ranks: Ranks) -> float:
    """Whole-job throughput: the units every rank processed over the time of
    the slowest rank."""
    return ranks.sum(units_per_rank) / ranks.max(seconds_per_rank)


def allreduce_mean_(tensors, ranks: Ranks | None):
    """Average ``tensors`` over all ranks in place with one flattened
    all-reduce (no-op on a single rank)."""
    if ranks is None or ranks.world == 1 or not tensors:
        return
    flat = torch.cat([t.reshape(-1) for t in tensors])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM)
    flat /= ranks.world
    off = 0
    for t in tensors:
        k = t.numel()
        t.copy_(flat[off:off + k].view_as(t))
        off += k


def global_moments(X, ranks: Ranks | None):
    """Column mean and (unbiased) standard deviation of the rows of ``X``
    gathered over all ranks: per-rank count, sum and sum of squares are
    all-reduced in FP64."""
    X64 = X.double()
    n = torch.tensor([float(X.shape[0])], dtype=torch.float64, device=X.device)
    s1, s2 = X64.sum(0), (X64 * X64).sum(0)
    if ranks is not None and ranks.world > 1:
        for t in (n, s1, s2):
            dist.all_reduce(t, op=dist.ReduceOp.SUM)
    N = n.item()
    mean = s1 / N
    var = ((s2 - N * mean * mean) / max(N - 1.0, 1.0)).clamp_min(0.0)
    return mean.to(X.dtype), var.sqrt().to(X.dtype)


def min_int(value: int, ranks: Ranks | None) -> int:
    """The smallest of every rank's ``value``."""
    if ranks is None or ranks.world == 1:
        return int(value)
    return int(ranks._reduce(float(value), dist.ReduceOp.MIN))
