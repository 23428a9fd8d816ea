"""One process per GPU: environment sharding and the scalar reductions of a
multi-GPU run.

Every LP instance is independent and the dFBA couples species only inside
one environment, so a multi-GPU run gives each rank its own environments
(weak scaling: a fixed number per GPU) and shares nothing on the data path.
The only collectives are scalar reductions for reporting: the maximum of the
per-rank device times (the job's time) and the sum of the per-rank counts.
``torch.distributed`` carries them (NCCL on GPUs, gloo on the CPU).
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
