"""Replica parallelism for independent traversals (one process per GPU).

A single traversal does not shard cheaply, but multi-source BFS / BC and
query streams are independent units: every rank holds the whole graph and
runs its own share of sources.  There is no data-path collective; ranks only
agree on timing (max over ranks) and on totals (sum over ranks).  These
helpers are backend-agnostic (NCCL on GPUs, gloo on CPU for tests)."""
from __future__ import annotations

import numpy as np


def shard(items, rank: int, world: int, per_rank: int | None = None) -> np.ndarray:
    """Contiguous share of `items` for `rank`.  With per_rank, every rank gets
    exactly that many (weak scaling: items must hold world * per_rank)."""
    items = np.asarray(items)
    if per_rank is not None:
        if items.size < world * per_rank:
            raise ValueError("not enough items for weak scaling")
        return items[rank * per_rank:(rank + 1) * per_rank]
    bounds = np.linspace(0, items.size, world + 1).astype(int)
    return items[bounds[rank]:bounds[rank + 1]]


def _reduce(value: float, op: str, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(value: float, device=None) -> float:
    """Job time = the slowest rank's time."""
    return _reduce(value, "max", device)


def sum_over_ranks(value: float, device=None) -> float:
    """Whole-job totals (edges traversed, queries served)."""
    return _reduce(value, "sum", device)


def whole_job_rate(units_per_rank: float, seconds_per_rank: float, device=None) -> float:
    """Units of all ranks divided by the max-over-ranks time."""
    return sum_over_ranks(units_per_rank, device) / max_over_ranks(seconds_per_rank, device)
