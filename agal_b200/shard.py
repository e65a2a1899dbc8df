"""Case sharding of independent-case batches across GPUs (one process per GPU).

The reference runs one case on one GPU (README.md:2; every ArgsPack has
N_DEV = 1), and a single case does not shard without a halo exchange the
reference does not have.  A batch of independent cases shards by case: each
rank builds and advances only its own cases, with no data-path collective;
the only collectives are the timing reductions (max of the ranks' device
times, sum of their cell updates).

Cases are packed by longest processing time first (LPT): sorted by cost,
each goes to the rank with the least cost so far (ties to the lowest rank),
which keeps the slowest rank within 4/3 of the optimum.  The cost of a case
is its work per coarse step: the cells of its base grid times 2^(levels-1),
since level L is stepped 2^L times per coarse step.
"""
from __future__ import annotations

import heapq
from typing import Sequence


def case_cost(spec: dict) -> float:
    """Work per coarse step of a batched case: base cells x 2^(levels-1)."""
    return float(spec["N"]) ** 3 * 2.0 ** (int(spec["levels"]) - 1)


def lpt_shards(costs: Sequence[float], n_ranks: int) -> list[list[int]]:
    """Case indices per rank, LPT-packed; each rank's list is in case order.
    Deterministic: equal costs keep their index order, equal loads go to the
    lower rank."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(n_ranks)]
    shards: list[list[int]] = [[] for _ in range(n_ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(s) for s in shards]


def shard_loads(costs: Sequence[float], shards: list[list[int]]) -> list[float]:
    return [sum(float(costs[i]) for i in s) for s in shards]


def aggregate(updates: float, ms: float, allsum, allmax) -> dict:
    """Whole-job throughput of a sharded batch: the cell updates of every
    rank over the slowest rank's device time (allsum / allmax reduce a float
    over the ranks)."""
    total = allsum(float(updates))
    slowest = allmax(float(ms))
    return {"cell_updates": total, "ms": slowest,
            "mlups": total / (slowest * 1e-3) / 1e6 if slowest > 0 else 0.0}
