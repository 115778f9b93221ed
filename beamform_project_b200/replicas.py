"""Independent replicas on N GPUs: one process per GPU under torchrun.

The beamformer path has no exchange step (channels, shards and served jobs
are independent), so N GPUs run N independent copies of a workload; the
process group only carries the barrier around the timed region and the
reductions of its result (the maximum time over ranks, the sum of work).
"""
from __future__ import annotations

import datetime
import os


class Replicas:
    def __init__(self, backend: str = "nccl", timeout_s: float = 120.0):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self._dist = None
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self._dist = dist

    def _reduce(self, value: float, op_name: str) -> float:
        if self._dist is None:
            return float(value)
        import torch
        dev = torch.device("cuda", self.local) if self.backend == "nccl" else torch.device("cpu")
        t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
        self._dist.all_reduce(t, op=getattr(self._dist.ReduceOp, op_name))
        return float(t.item())

    def max(self, value: float) -> float:
        """Maximum over ranks (the job time of a weak-scaling run)."""
        return self._reduce(value, "MAX")

    def sum(self, value: float) -> float:
        """Sum over ranks (the work all replicas did)."""
        return self._reduce(value, "SUM")

    def barrier(self) -> None:
        if self._dist is not None:
            self._dist.barrier()

    def close(self) -> None:
        if self._dist is not None:
            self._dist.destroy_process_group()
            self._dist = None

    @staticmethod
    def partition(n_items: int, rank: int, world: int) -> range:
        """Contiguous, balanced share of n_items for `rank` (sizes differ by at most one)."""
        base, extra = divmod(n_items, world)
        start = rank * base + min(rank, extra)
        return range(start, start + base + (1 if rank < extra else 0))
