"""Sharding of independent ensemble members (stochastic Heun runs, relaxation
samples) over the ranks of a ``torch.distributed`` process group.

Members are independent: each rank runs the members assigned to it on its own
GPU, and the only collective is one gather of the per-member results at the
end.  The assignment is static and cost-balanced (longest-processing-time
first over cost = cells x steps), identical on every rank because it is a pure
function of the member list.  A member that raises on one rank does not leave
the others waiting: every rank still takes part in the gather, and afterwards
all ranks raise the same error naming the failed members.
"""
from __future__ import annotations

import heapq
from typing import Any, Callable, List, Optional, Sequence


def assign(costs: Sequence[float], world_size: int) -> List[List[int]]:
    """Member indices per rank, longest-processing-time first: members sorted by
    decreasing cost (ties by index) go to the least-loaded rank (ties by rank)."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world_size)]
    out: List[List[int]] = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    for lst in out:
        lst.sort()
    return out


def member_cost(nx: int, ny: int, nz: int, steps: int) -> float:
    """Cost model of one member: cells x steps."""
    return float(nx) * ny * nz * steps


def run_sharded(members: Sequence[Any], costs: Sequence[float], run_member: Callable[[Any], Any],
                group: Optional[Any] = None) -> List[Any]:
    """Runs run_member(members[i]) for the members assigned to this rank and
    returns every member's result, in member order, on every rank.

    Without an initialised process group the call runs all members locally.
    """
    import torch.distributed as dist

    if len(members) != len(costs):
        raise ValueError("members and costs differ in length")
    if not (dist.is_available() and dist.is_initialized()):
        return [run_member(m) for m in members]
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    mine = assign(costs, world)[rank]
    local = []
    for i in mine:
        try:
            local.append((i, True, run_member(members[i])))
        except Exception as e:  # reported after the gather, on every rank
            local.append((i, False, "%s: %s" % (type(e).__name__, e)))
    gathered: List[Any] = [None] * world
    dist.all_gather_object(gathered, local, group=group)
    results: List[Any] = [None] * len(members)
    failed = []
    for part in gathered:
        for i, ok, value in part:
            if ok:
                results[i] = value
            else:
                failed.append((i, value))
    if failed:
        failed.sort()
        raise RuntimeError("ensemble members failed: " + "; ".join("member %d (%s)" % f for f in failed))
    return results
