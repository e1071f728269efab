"""Multi-GPU helpers: meshes and requests are independent units with no exchange, so N ranks
(one process per GPU) either run replicas or split the meshes, and only timings and results
meet on the host.

* ``balanced_partition`` assigns meshes to ranks, largest first, each to the rank with the
  fewest triangles so far (greedy longest-processing-time bin packing on triangle counts).
* ``reduce_max`` / ``gather_objects`` are the only collectives: the slowest rank's time and
  the host-side gather of results, over whatever backend the process group uses (NCCL on
  GPUs, gloo on CPU).
"""
from __future__ import annotations

import heapq
from typing import Sequence


def balanced_partition(sizes: Sequence[int], parts: int) -> list[list[int]]:
    """Indices of `sizes` per part, each part's total as even as the greedy rule makes it;
    indices within a part keep their input order."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    heap = [(0, r) for r in range(parts)]
    out: list[list[int]] = [[] for _ in range(parts)]
    for i in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(sizes[i]), r))
    return [sorted(p) for p in out]


def reduce_max(value: float, device=None) -> float:
    """The maximum of `value` over the ranks of the default process group (the value itself
    when no group is initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_objects(obj):
    """Every rank's `obj`, in rank order, on every rank."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out
