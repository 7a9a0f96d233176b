"""Sharding of independent solves over ranks (one process per GPU).

The configurations of this path shard into independent units: the momentum
sectors and scan points of a parameter scan, disorder instances of a quench,
benchmark replicas. Units are assigned by longest processing time on their
weights (dimensions), solved locally, and only their small results (eigen-
values, bounds) are gathered; no vector crosses ranks. A unit that fails on one
rank is reported on every rank after the same single gather, so all ranks take
the same collective steps on the error path too.
"""

from __future__ import annotations

import heapq
import traceback


def lpt_partition(weights, ranks: int) -> list[list[int]]:
    """Longest-processing-time assignment of units (by weight) to ranks.

    Units are taken heaviest first (ties by index); each goes to the rank with
    the least load so far (ties by rank). Deterministic."""
    if ranks < 1:
        raise ValueError("ranks must be positive")
    order = sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i))
    heap = [(0.0, r) for r in range(ranks)]
    heapq.heapify(heap)
    parts: list[list[int]] = [[] for _ in range(ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(weights[i]), r))
    return [sorted(p) for p in parts]


class ShardError(RuntimeError):
    """A unit failed on some rank; raised on every rank."""


def run_sharded(units, weights, solve, group=None) -> list:
    """Solve `units` over the ranks of `group` (torch.distributed) and return
    every unit's result, in unit order, on every rank.

    `solve(unit)` returns a picklable result. Without an initialised process
    group this runs serially."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return [solve(u) for u in units]
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    mine = lpt_partition(weights, world)[rank]
    local: dict[int, object] = {}
    failure = None
    for i in mine:
        try:
            local[i] = solve(units[i])
        except Exception as exc:  # reported after the gather, on every rank
            failure = (rank, i, f"{type(exc).__name__}: {exc}", traceback.format_exc())
            break
    gathered: list = [None] * world
    dist.all_gather_object(gathered, (local, failure), group=group)
    failures = [f for _, f in gathered if f is not None]
    if failures:
        r, i, message, _ = failures[0]
        raise ShardError(f"unit {i} failed on rank {r}: {message}")
    results: dict[int, object] = {}
    for part, _ in gathered:
        results.update(part)
    if sorted(results) != list(range(len(units))):
        raise ShardError("the gathered results do not cover every unit exactly once")
    return [results[i] for i in range(len(units))]
