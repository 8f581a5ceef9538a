"""Work split across GPUs (one process per GPU).

The reference runs one scenario on one GPU and has no communication.  Here
independent units shard with no collective in the data path:
  * an ensemble of scenarios is split across ranks by particle count
    (longest-processing-time greedy bin packing), each rank running its
    share as one batched simulation;
  * a single large scenario is replicated (each rank runs its own copy).
torch.distributed is only used around the timed region: a barrier before
it and a max-reduction of the device time after it.
"""
from __future__ import annotations

import heapq


def partition(counts, world: int):
    """Splits units with the given work `counts` over `world` ranks, largest
    first onto the least-loaded rank.  Returns one sorted list of unit
    indices per rank; every unit appears exactly once."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    shares = [[] for _ in range(world)]
    for k in sorted(range(len(counts)), key=lambda k: (-counts[k], k)):
        load, r = heapq.heappop(heap)
        shares[r].append(k)
        heapq.heappush(heap, (load + float(counts[k]), r))
    return [sorted(s) for s in shares]


def imbalance(counts, shares) -> float:
    """Largest rank load over the mean load (1.0 is perfect balance)."""
    loads = [sum(counts[k] for k in s) for s in shares]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean > 0 else 1.0


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over all ranks (the value itself without an
    initialised process group)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
