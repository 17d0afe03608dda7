"""World shards across ranks: one process per GPU, each stepping its own
worlds with no data-path collective (worlds never interact).  The only
collectives are the barrier around a timed region and the max-over-ranks
reduction of its duration; the whole-job throughput is every rank's worlds
over that maximum.  Works over NCCL (CUDA tensors) and gloo (CPU tensors),
so the multi-rank logic is testable without a GPU."""

from __future__ import annotations

import os
from dataclasses import dataclass


@dataclass(frozen=True)
class Shard:
    rank: int
    world_size: int
    worlds: int  # worlds on this rank
    first_world: int  # global index of this rank's first world
    seed: int  # scene seed of this rank (distinct per rank)


def shard_of(rank: int, world_size: int, worlds_per_rank: int, base_seed: int) -> Shard:
    """Weak scaling: every rank holds `worlds_per_rank` worlds of its own,
    seeded base_seed + 1000 * rank."""
    if not (0 <= rank < world_size):
        raise ValueError(f"rank {rank} outside world size {world_size}")
    return Shard(rank, world_size, int(worlds_per_rank), rank * int(worlds_per_rank), int(base_seed) + 1000 * rank)


def env_ranks() -> tuple[int, int, int]:
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class RankGroup:
    """Barrier and max-over-ranks timing for a process group (or none: one
    rank).  `device` is where the reduction tensor lives: the rank's GPU for
    NCCL, the CPU for gloo."""

    def __init__(self, dist=None, device=None):
        self.dist = dist
        self.device = device

    def _cuda(self) -> bool:
        return self.device is not None and getattr(self.device, "type", str(self.device)) == "cuda"

    def barrier(self) -> None:
        import torch

        if self.dist is not None:
            self.dist.barrier()
        if self._cuda():
            torch.cuda.synchronize(self.device)

    def max_over_ranks(self, x: float) -> float:
        import torch

        if self.dist is None:
            return float(x)
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(self, x: float) -> float:
        import torch

        if self.dist is None:
            return float(x)
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())


def job_throughput(worlds_per_rank: int, world_size: int, ms_max: float) -> float:
    """World-steps per second of the whole job: all ranks' worlds over the
    slowest rank's milliseconds per step."""
    if not ms_max > 0.0:
        raise ValueError("a timed step must take positive time")
    return worlds_per_rank * world_size / (ms_max * 1e-3)
