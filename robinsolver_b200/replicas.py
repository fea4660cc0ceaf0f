"""Replica plumbing for runs on N GPUs of one node.

The factor/solve path does not shard: every rank (one process per GPU, launched by torchrun)
factors and solves its own copy of the workload, and no collective touches the data path.  What
ranks share is only the bracketing of a timed region (a barrier on both sides), the maximum of
their device-timed durations, and the whole-job rate computed from it: N ranks x units per rank
/ the slowest rank's time (weak scaling).  The same class runs over NCCL on GPUs and over gloo
on CPU, which is how the multi-rank path is tested without GPUs.
"""
from __future__ import annotations

import os
from datetime import timedelta


class Replicas:
    """Process-group membership of one replica; a single process needs no group at all."""

    def __init__(self, backend: str = "nccl", device=None, timeout_s: float = 300.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.device = device
        self._dist = None
        if self.world > 1:
            import torch.distributed as dist
            kw = {"timeout": timedelta(seconds=timeout_s)}
            if backend == "nccl" and device is not None:
                kw["device_id"] = device
            dist.init_process_group(backend, **kw)
            self._dist = dist

    @property
    def leader(self) -> bool:
        """Rank 0 prints the result line."""
        return self.rank == 0

    def barrier(self) -> None:
        if self._dist is not None:
            self._dist.barrier()

    def max(self, x: float) -> float:
        """Maximum of x over all ranks (x itself for one process)."""
        if self._dist is None:
            return float(x)
        import torch
        dev = self.device if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def rate(self, units_per_rank: float, ms_local: float) -> tuple[float, float]:
        """(whole-job units per second, slowest rank's ms): every rank processed units_per_rank."""
        ms = self.max(ms_local)
        return self.world * units_per_rank / (ms * 1e-3), ms

    def close(self) -> None:
        if self._dist is not None:
            self._dist.destroy_process_group()
            self._dist = None
