"""Replicas across GPUs: every rank holds the whole index and searches its own
shard of the queries; no collective runs on the search path. The only
exchanges are host-side bookkeeping: a barrier around the timed region, the
maximum of the per-rank device times, and the operating point chosen on
rank 0 (torch.distributed: NCCL on GPUs, gloo on CPUs).
"""
from __future__ import annotations

import os


def env():
    """(rank, world_size, local_rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(rank: int, per_rank: int) -> slice:
    """Rows of rank `rank` in a query set of world * per_rank rows (weak scaling)."""
    return slice(rank * per_rank, (rank + 1) * per_rank)


class Ranks:
    def __init__(self, world: int, device=None):
        self.world = world
        self.device = device

    def _dist(self):
        import torch.distributed as dist
        return dist

    def barrier(self):
        if self.world > 1:
            self._dist().barrier()

    def max(self, x: float) -> float:
        if self.world == 1:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self._dist().all_reduce(t, op=self._dist().ReduceOp.MAX)
        return float(t.item())

    def broadcast_ints(self, values, src: int = 0):
        if self.world == 1:
            return list(values)
        import torch
        t = torch.tensor(list(values), dtype=torch.int64, device=self.device)
        self._dist().broadcast(t, src)
        return [int(x) for x in t.tolist()]

    def broadcast_json(self, obj, src: int = 0):
        """A JSON-serialisable object from rank `src` to every rank."""
        if self.world == 1:
            return obj
        box = [obj]
        self._dist().broadcast_object_list(box, src)
        return box[0]
