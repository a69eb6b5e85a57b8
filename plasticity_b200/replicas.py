"""Replica plumbing for runs on N GPUs of one node (one process per GPU).

The path does not shard: every rank solves its own copy of the workload
(independent replicas), and the only collectives are a barrier around timed
regions and the maximum of the ranks' times.  ``bench.py`` uses the NCCL
backend on the GPUs; the same functions run with gloo on the CPU in the tests.
"""
from __future__ import annotations

import os
from datetime import timedelta


class Replicas:
    """Rank layout from the launcher's environment (RANK, WORLD_SIZE,
    LOCAL_RANK) and, for world > 1, a process group with a short timeout so
    that ranks waiting for a missing peer end with an error."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 120.0):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch
            import torch.distributed as td
            kw = {}
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                kw["device_id"] = torch.device("cuda", self.local)
            td.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)
            self.dist = td

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max_over_ranks(self, x: float) -> float:
        """The largest of the ranks' values (every rank gets it)."""
        if not self.dist:
            return x
        import torch
        dev = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None
