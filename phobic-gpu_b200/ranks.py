"""One process per GPU: rank bookkeeping for builds that shard across GPUs.

An MPHF build partitions its keys into independent partitions and the reference
builds on one device (MPHFbuilder, include/phobicGpu/mphf_builder.h).  Across
GPUs the work therefore shards without any data exchange: every rank builds its
own key set (replicas of the build, weak scaling) or its own shard of one key set
(`shard_range`), and the only collectives are the barrier and the max-over-ranks
of the timings.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass(frozen=True)
class RankInfo:
    world: int
    rank: int
    local: int

    @staticmethod
    def from_env() -> "RankInfo":
        return RankInfo(int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
                        int(os.environ.get("LOCAL_RANK", "0")))


class Group:
    """The process group of a multi-rank run (None-safe: a world of one needs no group).

    backend "nccl" for GPU runs, "gloo" for CPU tests.  The timeout is short so that
    ranks waiting on a rank that left end with an error instead of hanging."""

    def __init__(self, info: RankInfo, backend: str = "nccl", timeout_s: float = 120.0, device=None):
        self.info = info
        self.device = device
        self.dist = None
        if info.world > 1:
            import torch.distributed as dist

            if not dist.is_initialized():
                dist.init_process_group(backend, rank=info.rank, world_size=info.world,
                                        timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self) -> None:
        if self.dist:
            self.dist.barrier()

    def max(self, x: float) -> float:
        """Largest x over all ranks (device times are reported as the slowest rank's)."""
        if not self.dist:
            return float(x)
        import torch

        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.dist:
            return float(x)
        import torch

        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self) -> None:
        if self.dist:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def rank_seed(seed: int, rank: int) -> int:
    """Seed of a rank's own key set: distinct ranks build distinct, independent sets."""
    return seed + rank


def shard_range(n: int, world: int, rank: int) -> tuple[int, int]:
    """[lo, hi) of rank's contiguous shard of n keys; shards are disjoint and cover [0, n)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank out of range")
    q, r = divmod(n, world)
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)
