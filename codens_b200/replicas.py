"""Replica runs over the GPUs of one node.

The hot path shards by independent cases, not by a collective: every rank
(one process per GPU, launched by torchrun) runs its own case on its own
GPU and no data crosses NVLink.  The ranks only meet to start the timed
region together and to agree on its length, which is the slowest rank's;
the whole-job rate is then every rank's work over that time (weak scaling).
"""
from __future__ import annotations

import datetime
import os


class Replicas:
    def __init__(self, backend: str = "nccl", timeout_s: float = 300.0):
        import torch
        import torch.distributed as dist
        self.torch, self.dist = torch, dist
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.device = "cuda" if backend == "nccl" else "cpu"
        if self.world > 1 and not dist.is_initialized():
            dist.init_process_group(backend, init_method="env://",
                                    timeout=datetime.timedelta(seconds=timeout_s))

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, x: float) -> float:
        """the largest x over the ranks (every rank gets it)"""
        t = self.torch.tensor([float(x)], dtype=self.torch.float64, device=self.device)
        if self.world > 1:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def rate(self, units_per_rank: float, seconds: float) -> float:
        """whole-job units per second: every rank's units over the slowest
        rank's time"""
        return self.world * units_per_rank / self.max(seconds)

    def close(self):
        if self.world > 1 and self.dist.is_initialized():
            self.dist.destroy_process_group()
