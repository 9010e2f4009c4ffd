"""Sharding of independent graphs across GPUs (batched and serving forms).

Graphs never share an SCC, so the batched form spreads them over ranks with
no data-path collective: every rank computes the same plan from the graphs'
byte sizes, builds and runs only its own shard, and the per-graph results
come back to the host side with one gather of Python objects (counts and,
optionally, label arrays that are already in host memory).  No counterpart
in the reference, which runs one graph per process.
"""
from __future__ import annotations

import heapq
from typing import Any, Callable, List, Optional, Sequence


def shard_by_bytes(nbytes: Sequence[int], world: int) -> List[List[int]]:
    """Greedy longest-processing-time bin packing: graphs in decreasing size
    order, each onto the rank with the fewest bytes so far (ties to the lower
    rank; equal sizes keep their index order).  Deterministic, so every rank
    computes the same plan.  Returns, per rank, its graph indices in
    increasing order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(nbytes)), key=lambda i: (-int(nbytes[i]), i))
    heap = [(0, r) for r in range(world)]
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(nbytes[i]), r))
    return [sorted(x) for x in out]


def gather_in_order(local: Sequence[Any], plan: List[List[int]], rank: int, group=None,
                    dst: Optional[int] = None) -> Optional[List[Any]]:
    """Reassembles per-graph results in global graph order.

    local: this rank's results, in the order of plan[rank].  With dst=None
    every rank receives the whole list (all_gather_object); otherwise only
    rank dst does and the others get None.  A world of 1 needs no process
    group.
    """
    world = len(plan)
    if len(local) != len(plan[rank]):
        raise ValueError("local results do not match this rank's shard")
    if world == 1:
        parts = [list(local)]
    else:
        import torch.distributed as dist
        if dst is None:
            parts = [None] * world
            dist.all_gather_object(parts, list(local), group=group)
        else:
            parts = [None] * world if rank == dst else None
            dist.gather_object(list(local), parts, dst=dst, group=group)
            if rank != dst:
                return None
    out: List[Any] = [None] * sum(len(p) for p in plan)
    for r in range(world):
        if len(parts[r]) != len(plan[r]):
            raise RuntimeError(f"rank {r} returned {len(parts[r])} results for {len(plan[r])} graphs")
        for i, res in zip(plan[r], parts[r]):
            out[i] = res
    return out


def run_sharded(nbytes: Sequence[int], build: Callable[[int], Any], solve: Callable[[List[Any]], List[Any]],
                rank: int, world: int, group=None, dst: Optional[int] = None) -> Optional[List[Any]]:
    """Plans the shards, builds this rank's graphs (build(i) for each of its
    indices), solves them in one call (solve(list) -> list of results) and
    gathers the results in global order."""
    plan = shard_by_bytes(nbytes, world)
    mine = [build(i) for i in plan[rank]]
    return gather_in_order(solve(mine), plan, rank, group=group, dst=dst)
