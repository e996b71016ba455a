"""Independent disks across GPUs: one process per GPU, no collective in the
data path.

A disk's work per step is its cell count (all stages scale with it), so a
set of disks is split over ranks by the longest-processing-time greedy rule:
heaviest disk first, each to the currently lightest rank.  Every rank
computes the same split from the same list.  The only collectives are the
ones around the measurement: a barrier and the maximum of the per-rank times
(torch.distributed; NCCL on GPUs, gloo on CPU)."""
from __future__ import annotations

import heapq
from typing import List, Sequence


def lpt_shards(costs: Sequence[float], world: int) -> List[List[int]]:
    """Indices of `costs` per rank (0..world-1), LPT greedy; ties go to the
    lower rank, so the split is deterministic."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0.0, r) for r in range(world)]
    out: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    for o in out:
        o.sort()
    return out


def shard_disks(cfgs, rank: int, world: int):
    """This rank's disks of a global list (LPT on active cells)."""
    idx = lpt_shards([c.active_cells * c.nfluids for c in cfgs], world)[rank]
    return [cfgs[i] for i in idx]


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank float over the default process group (the
    identity without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
