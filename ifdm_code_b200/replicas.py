"""Replica plumbing for several GPUs: one independent box per rank.

The leap-frog path does not shard (a box is advanced on one GPU), so several
GPUs run independent replicas: no data crosses between ranks.  The process
group is used only for the barriers around the timed region and for taking
the maximum of the ranks' times, so the whole job's throughput is
world x (cells x steps) / max-over-ranks time.  Ranks come from the torchrun
environment (RANK, LOCAL_RANK, WORLD_SIZE, MASTER_ADDR, MASTER_PORT); NCCL on
GPUs, gloo on CPU (tests).
"""

from __future__ import annotations

import datetime
import os


class Replicas:
    def __init__(self, backend: str | None = None, timeout_s: float = 600.0):
        import torch

        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        self.cuda = self.backend == "nccl"
        self.dist = None
        if self.cuda:
            torch.cuda.set_device(self.local)
        if self.world > 1:
            import torch.distributed as dist

            dist.init_process_group(self.backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self) -> None:
        import torch

        if self.dist:
            self.dist.barrier()
        if self.cuda:
            torch.cuda.synchronize()

    def max(self, v: float) -> float:
        """The maximum of v over all ranks (every rank gets it)."""
        import torch

        if not self.dist:
            return float(v)
        t = torch.tensor([float(v)], dtype=torch.float64, device="cuda" if self.cuda else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def throughput(self, units_per_rank: float, seconds_max: float) -> float:
        """Whole-job rate: every rank processed units_per_rank in at most seconds_max."""
        return self.world * units_per_rank / seconds_max

    def close(self) -> None:
        if self.dist:
            self.dist.destroy_process_group()
            self.dist = None
