"""Replica plumbing for one process per GPU.

The fit does not shard in the reference (one GPU, one process), so N GPUs run N independent
replicas of the whole workload: every rank owns its context and device, and the only
collective steps are barriers around a timed region and the maximum of the ranks' times,
from which the whole-job throughput is N * steps / max_time. Ranks, world size and the
rendezvous come from the torchrun environment (RANK, LOCAL_RANK, WORLD_SIZE, MASTER_ADDR,
MASTER_PORT). The backend is NCCL on GPUs; gloo serves the CPU tests of this logic.
"""
from __future__ import annotations

import datetime
import os


class Replicas:
    def __init__(self, backend: str = "nccl", timeout_s: float = 600.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist

            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def _device(self):
        return f"cuda:{self.local}" if self.backend == "nccl" else "cpu"

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()

    def max_time(self, seconds: float) -> float:
        """The largest of the ranks' times (every rank gets it)."""
        if self.dist is None:
            return float(seconds)
        import torch

        t = torch.tensor([float(seconds)], dtype=torch.float64, device=self._device())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def throughput(self, steps: int, seconds: float) -> float:
        """Whole-job rate: all ranks' steps over the slowest rank's time."""
        return self.world * steps / self.max_time(seconds)

    def close(self) -> None:
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None
