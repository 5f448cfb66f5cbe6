"""Multi-GPU bookkeeping for the transform: replicas, not a partitioned solve.

Field-levels are independent, so N GPUs run N independent batches with no data
exchange.  The only collectives are a barrier around the timed region and the
reductions of the timing: the max of the device time over ranks, and the
sum of the work.  One process per GPU; RANK, LOCAL_RANK and WORLD_SIZE come from
the launcher (torchrun), rendezvous on 127.0.0.1.
"""
from __future__ import annotations

import os
from datetime import timedelta


def world_info():
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Replicas:
    """Barrier and timing reductions over the ranks of one job.

    backend: "nccl" for GPU runs (reductions on a CUDA tensor), "gloo" on CPU.
    A short process-group timeout ends a collective with an error when a rank
    is missing instead of waiting forever.
    """

    def __init__(self, backend: str = "nccl", device=None, timeout_s: float = 120.0):
        import torch
        import torch.distributed as dist

        self.world, self.rank, self.local_rank = world_info()
        self.backend = backend
        self.device = device if backend == "nccl" else torch.device("cpu")
        self._dist = dist
        self._torch = torch
        self.active = self.world > 1
        if self.active and not dist.is_initialized():
            kw = dict(backend=backend, timeout=timedelta(seconds=timeout_s))
            if backend == "nccl" and device is not None:
                kw["device_id"] = device
            dist.init_process_group(**kw)

    def barrier(self):
        if self.active:
            self._dist.barrier()

    def _reduce(self, x: float, op) -> float:
        if not self.active:
            return float(x)
        t = self._torch.tensor([float(x)], dtype=self._torch.float64, device=self.device)
        self._dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        return self._reduce(x, self._dist.ReduceOp.MAX)

    def sum(self, x: float) -> float:
        return self._reduce(x, self._dist.ReduceOp.SUM)

    def throughput(self, units_per_rank: float, seconds_on_rank: float) -> float:
        """Whole-job units per second: every rank's units over the slowest rank's time."""
        return self.sum(units_per_rank) / self.max(seconds_on_rank)

    def close(self):
        if self.active and self._dist.is_initialized():
            self._dist.destroy_process_group()
