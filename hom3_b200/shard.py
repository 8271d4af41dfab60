"""Sharding independent grids (batch instances) across ranks.

The batched workload is a set of independent grids: nothing couples two
instances, so the natural multi-GPU split gives each rank (one process per
GPU) a share of the instances, which it steps as one batch (h3c_set_grids)
with no collective on the data path.  Only the results are gathered at the
end.  hom3 itself has no domain decomposition (it is serial), so there is
no reference behaviour to match beyond "each instance evolves exactly as it
would alone", which the gather lets a caller check.

partition() balances the leaf-cell counts over the ranks (longest
processing time first, deterministic: ties go to the lower rank and the
lower instance index), and gather() collects per-instance results on every
rank in the original instance order through torch.distributed (gloo on CPU,
NCCL between GPUs).
"""
from __future__ import annotations

import heapq
from typing import Any, List, Sequence


def partition(cells: Sequence[int], world_size: int) -> List[List[int]]:
    """Instance indices per rank, each rank's list ascending, so that the
    largest per-rank leaf-cell total is small (greedy: instances in
    decreasing size to the currently lightest rank)."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(cells)), key=lambda i: (-int(cells[i]), i))
    heap = [(0, r) for r in range(world_size)]
    out: List[List[int]] = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(cells[i]), r))
    return [sorted(x) for x in out]


def gather(local: Sequence[Any], assignment: List[List[int]], rank: int, group=None) -> List[Any]:
    """Every rank passes the results of its own instances (in the order of
    assignment[rank]); every rank gets all instances' results in instance
    order.  With one rank no collective is made."""
    n = sum(len(a) for a in assignment)
    if len(assignment) == 1:
        return list(local)
    import torch.distributed as dist
    if len(local) != len(assignment[rank]):
        raise ValueError("rank %d holds %d results for %d instances" % (rank, len(local), len(assignment[rank])))
    parts: List[Any] = [None] * len(assignment)
    dist.all_gather_object(parts, list(local), group=group)
    out: List[Any] = [None] * n
    for r, idx in enumerate(assignment):
        for k, i in enumerate(idx):
            out[i] = parts[r][k]
    return out
