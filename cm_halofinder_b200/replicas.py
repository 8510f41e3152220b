"""One box per GPU: the plumbing of multi-GPU runs.

Boxes, lightcone shells and batches are independent domains, so the ranks
of a run exchange nothing but a few scalars: each rank (one process per
GPU, launched by torchrun) runs FoF on its own domains, times its steps on
its own device, and the run reports the slowest rank's time and the total
of the particles (weak scaling).  This module holds that plumbing so that
it can be exercised with the gloo backend on CPU as well as with NCCL.
"""
from __future__ import annotations

import datetime
import os


class Replicas:
    """Rank layout from the torchrun environment and the few collectives a
    replica run needs.  With WORLD_SIZE 1 nothing is initialised."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 600.0):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        self.device = None
        if backend == "nccl":
            import torch
            torch.cuda.set_device(self.local)
            self.device = torch.device("cuda", self.local)
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def _tensor(self, x):
        import torch
        return torch.tensor([float(x)], dtype=torch.float64,
                            device=self.device if self.device is not None else "cpu")

    def barrier(self):
        """All ranks here, and this rank's device idle."""
        if self.dist is not None:
            self.dist.barrier()
        if self.device is not None:
            import torch
            torch.cuda.synchronize(self.device)

    def max(self, x: float) -> float:
        """Largest x over the ranks (a step time: the slowest rank)."""
        if self.dist is None:
            return float(x)
        t = self._tensor(x)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        """Total of x over the ranks (particles processed)."""
        if self.dist is None:
            return float(x)
        t = self._tensor(x)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    @staticmethod
    def share(nbox: int, rank: int, world: int) -> list[int]:
        """Boxes of one rank when `nbox` boxes are dealt round-robin."""
        return list(range(rank, nbox, world))

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None
