"""Independent replicas over ranks: one process per GPU, no collective on the data path.

A tessellation does not shard usefully below one structure (the work per structure is
local and small next to a halo exchange), so several GPUs run independent structures:
each rank tessellates its own inputs, and the only collectives are the barriers around
the timed region and the max-over-ranks of the measured times.  The structures of one
batch are split into contiguous blocks, one per rank, of about equal ball counts
(``partition_weighted``): each rank runs its block as one batched call.

``Ranks`` reads RANK / WORLD_SIZE / LOCAL_RANK from the environment (torchrun) and joins a
process group when WORLD_SIZE > 1 (``nccl`` on GPUs; ``gloo`` for the CPU tests).
"""
from __future__ import annotations

import datetime
import os


def partition(count: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous block [start, stop) of `count` items for `rank` of `world` ranks; block
    sizes differ by at most one and the blocks cover every item exactly once."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world / rank")
    base, extra = divmod(count, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def partition_weighted(weights, world: int, rank: int) -> tuple[int, int]:
    """Contiguous block [start, stop) of the items for `rank` of `world` ranks, cut where
    the running sum of `weights` (e.g. balls per structure) crosses k / world of the
    total, so every rank gets about the same weight; the blocks cover every item exactly
    once, in order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world / rank")
    import numpy as np

    w = np.asarray(weights, dtype=np.float64)
    if len(w) == 0:
        return 0, 0
    c = np.cumsum(w)
    total = c[-1]

    def cut(k):
        if k <= 0:
            return 0
        if k >= world:
            return len(w)
        return int(np.searchsorted(c, total * k / world, side="left")) + 1

    start, stop = cut(rank), cut(rank + 1)
    return min(start, len(w)), min(max(stop, start), len(w))


def replica_throughput(units_per_rank: float, world: int, max_ms: float) -> float:
    """Whole-job throughput of `world` replicas that each processed `units_per_rank` units,
    timed as the slowest rank (max over ranks, in milliseconds)."""
    return world * units_per_rank / (max_ms * 1e-3)


class Ranks:
    def __init__(self, backend: str = "nccl", timeout_s: float = 120.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist

            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def _device(self):
        return "cuda" if self.backend == "nccl" else "cpu"

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()
        if self.backend == "nccl":
            import torch

            torch.cuda.synchronize()

    def max(self, x: float) -> float:
        """Maximum of x over all ranks (every rank calls it, in the same order)."""
        if self.dist is None:
            return float(x)
        import torch

        t = torch.tensor([float(x)], dtype=torch.float64, device=self._device())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self) -> None:
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None
