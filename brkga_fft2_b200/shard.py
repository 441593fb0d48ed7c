"""Multi-GPU plumbing: one process per GPU, the population split by rows.

The decode shards without any exchange: every (chromosome, machine) item is
independent, so each rank decodes its own rows.  The only collective a GA
needs is an all-gather of the P float64 makespans before ranking (and, for
timing, a max over ranks).  ``torch.distributed`` carries both (NCCL on GPUs,
gloo in the CPU tests).
"""
from __future__ import annotations

from typing import Callable, List, Optional, Tuple


def row_range(total: int, rank: int, world: int) -> Tuple[int, int]:
    """Rows [start, end) of rank in a population of `total` split as evenly as possible."""
    if world < 1 or not 0 <= rank < world or total < 0:
        raise ValueError("bad rank/world/total")
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def rank_seed(rank: int, step: int) -> int:
    """Seed of the population a rank decodes at a given step (weak scaling: distinct per rank)."""
    return 1_000_003 * (rank + 1) + step


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Max of a float over all ranks (identity without a process group)."""
    if dist is None or not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_throughput(units_per_rank: int, world: int, max_seconds: float) -> float:
    """Whole-job units per second when every rank processes the same amount."""
    return units_per_rank * world / max_seconds


class ShardedDecode:
    """Decode a population replicated on every rank: each rank decodes its row
    range with `decode_rows(rows) -> makespans`, then all ranks all-gather the
    makespans so every rank holds the full fitness vector (the exchange a
    multi-GPU GA needs before ranking)."""

    def __init__(self, decode_rows: Callable, dist=None):
        self.decode_rows = decode_rows
        self.dist = dist

    def __call__(self, population):
        import torch
        dist = self.dist
        world = dist.get_world_size() if dist is not None and dist.is_initialized() else 1
        rank = dist.get_rank() if world > 1 else 0
        P = population.shape[0]
        start, end = row_range(P, rank, world)
        local = self.decode_rows(population[start:end])
        local = torch.as_tensor(local, dtype=torch.float64, device=population.device)
        if world == 1:
            return local
        # all-gather with equal-size buffers (ranks differ by at most one row)
        width = -(-P // world)
        buf = torch.full((width,), float("nan"), dtype=torch.float64, device=population.device)
        buf[: end - start] = local
        parts: List = [torch.empty_like(buf) for _ in range(world)]
        dist.all_gather(parts, buf)
        out = []
        for r in range(world):
            s, e = row_range(P, r, world)
            out.append(parts[r][: e - s])
        return torch.cat(out)
