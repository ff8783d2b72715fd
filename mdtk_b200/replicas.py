"""Independent replicas, one process per GPU (the path does not shard: each
rank advances its own trajectory; there is no data-path collective).

The launcher (torchrun) sets RANK / LOCAL_RANK / WORLD_SIZE / MASTER_*;
with WORLD_SIZE 1 nothing is initialised.  The only collectives are the
barrier around a timed region and the maximum of the ranks' device times,
so the reported time is that of the slowest replica."""
from __future__ import annotations

import os
from datetime import timedelta


class Replicas:
    def __init__(self, backend: str = "nccl", timeout_s: float = 300.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch
            import torch.distributed as dist
            kw = {}
            if backend == "nccl":
                kw["device_id"] = torch.device("cuda", self.local)
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x: float) -> float:
        """The largest x over the ranks (every rank gets it)."""
        if self.dist is None:
            return float(x)
        import torch
        dev = torch.device("cuda", self.local) if self.backend == "nccl" else torch.device("cpu")
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


def aggregate_rate(units_per_rank: float, world: int, max_seconds: float) -> float:
    """Whole-job throughput: the units all ranks processed over the slowest
    rank's time (weak scaling: every rank processes units_per_rank)."""
    return world * units_per_rank / max_seconds
