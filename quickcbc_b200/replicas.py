"""One process per GPU, each an independent replica of the likelihood workload.

Parameter sets and events are independent units with no exchange step, so
replicas share nothing on the data path; the only cross-rank traffic is the
barrier around a timed region and the max-over-ranks reduction of its duration.
That plumbing runs over torch.distributed's gloo backend on host tensors, so it
works (and is tested) without GPUs.
"""
from __future__ import annotations

import os


class Replicas:
    def __init__(self):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", str(self.rank)))
        self._dist = None
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            if not dist.is_initialized():
                dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=120))
            self._dist = dist

    @property
    def is_root(self) -> bool:
        return self.rank == 0

    def barrier(self):
        if self._dist:
            self._dist.barrier()

    def max_over_ranks(self, value: float) -> float:
        if not self._dist:
            return float(value)
        import torch
        t = torch.tensor([float(value)], dtype=torch.float64)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(self, value: float) -> float:
        if not self._dist:
            return float(value)
        import torch
        t = torch.tensor([float(value)], dtype=torch.float64)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM)
        return float(t.item())

    def seed_offset(self) -> int:
        """Each replica draws its own parameter sets."""
        return self.rank

    def close(self):
        if self._dist and self._dist.is_initialized():
            self._dist.destroy_process_group()
        self._dist = None
