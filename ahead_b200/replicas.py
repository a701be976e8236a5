"""Process-group plumbing of a multi-GPU run: one process per GPU, each holding
a full replica of the resident schema and serving its own query stream.  The
query path has no exchange step between replicas (no collective on the data
path); the only collectives are the barriers around the timed region and the
maximum of the per-rank times (the job's time), plus sums of per-rank counts.
"""
from __future__ import annotations

import datetime
import os


class Replicas:
    """torch.distributed over the ranks of this job (one per GPU), or a
    single process when WORLD_SIZE is 1 / unset."""

    def __init__(self, backend: str = "nccl", timeout_s: int = 300):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self._dist = None
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self._dist = dist

    def _tensor(self, x: float):
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        return torch.tensor([float(x)], dtype=torch.float64, device=dev)

    def barrier(self):
        if self._dist is not None:
            self._dist.barrier()

    def max(self, x: float) -> float:
        """The largest value over ranks (the job's time of a timed region)."""
        if self._dist is None:
            return float(x)
        t = self._tensor(x)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if self._dist is None:
            return float(x)
        t = self._tensor(x)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM)
        return float(t.item())

    def seed(self, seed: int) -> int:
        """The query-stream seed of this replica (different streams per rank)."""
        return seed + 1000 * self.rank

    def close(self):
        if self._dist is not None:
            self._dist.barrier()
            self._dist.destroy_process_group()
            self._dist = None
