"""Partitioning of a batch of independent factorizations over the ranks of a job.

Instances of a pattern are independent (one symbolic analysis, many value sets), so a batch
shards with no data-path exchange: every rank holds its own copy of the plan and factors its own
share of the instances.  The reference runs one factorization on device 0 only
(src/numeric.cu:344-346); this module is what spreads a batch over several GPUs.

* :func:`instance_range` -- one pattern: a contiguous, balanced block of the batch per rank.
* :func:`plan_shards` -- several patterns of uneven cost (the multi-pattern batch): every
  pattern's instances are cut into chunks of about equal cost, the chunks are assigned longest
  first to the least-loaded rank (LPT), and a rank's chunks of one pattern are merged back into
  contiguous ranges.  The cost of an instance is its pattern's algorithmic flop count F_alg.
* :func:`instance_seeds` -- per-instance value seeds, so an instance's values depend only on its
  global index and the union of the shards is exactly the batch, whatever the rank count.

Every rank computes the same assignment from the same inputs (no communication).
"""
from __future__ import annotations

import dataclasses
import heapq


def instance_range(total: int, world: int, rank: int) -> tuple[int, int]:
    """(first, count) of rank ``rank``'s block of a batch of ``total`` instances: the first
    ``total % world`` ranks take one instance more."""
    if world < 1 or not 0 <= rank < world or total < 0:
        raise ValueError("need world >= 1, 0 <= rank < world, total >= 0")
    base, extra = divmod(total, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


@dataclasses.dataclass(frozen=True)
class Shard:
    """Instances [first, first + count) of pattern ``name`` on one rank."""
    name: str
    first: int
    count: int


def plan_shards(patterns: list[tuple[str, int, float]], world: int,
                chunks_per_rank: int = 4) -> list[list[Shard]]:
    """Assigns the instances of several patterns to ``world`` ranks, balanced by cost.

    ``patterns``: (name, instances, cost per instance).  Returns, per rank, its shards (at most one
    contiguous range per pattern run of chunks; patterns in input order).  Each pattern's batch is
    cut into chunks of about ``total_cost / (world * chunks_per_rank)`` (at least one instance
    each), then the chunks go, most expensive first, to the rank with the least cost so far (ties:
    the lower rank).  The result covers every (pattern, instance) exactly once.
    """
    if world < 1:
        raise ValueError("world must be >= 1")
    total = sum(cnt * cost for _, cnt, cost in patterns)
    target = total / (world * max(1, chunks_per_rank)) if total > 0 else 1.0
    chunks = []                                  # (cost, pattern index, first, count)
    for pi, (name, cnt, cost) in enumerate(patterns):
        if cnt <= 0:
            continue
        per = max(1, int(target // cost)) if cost > 0 else cnt
        nchunk = -(-cnt // per)
        for k in range(nchunk):
            first, c = instance_range(cnt, nchunk, k)
            chunks.append((c * cost, pi, first, c))
    chunks.sort(key=lambda t: (-t[0], t[1], t[2]))
    heap = [(0.0, r) for r in range(world)]
    assigned: list[list[tuple[int, int, int]]] = [[] for _ in range(world)]
    for cost, pi, first, c in chunks:
        load, r = heapq.heappop(heap)
        assigned[r].append((pi, first, c))
        heapq.heappush(heap, (load + cost, r))
    out = []
    for r in range(world):
        parts = sorted(assigned[r])
        merged: list[Shard] = []
        for pi, first, c in parts:
            name = patterns[pi][0]
            if merged and merged[-1].name == name and merged[-1].first + merged[-1].count == first:
                last = merged.pop()
                merged.append(Shard(name, last.first, last.count + c))
            else:
                merged.append(Shard(name, first, c))
        out.append(merged)
    return out


def shard_cost(shards: list[Shard], cost: dict[str, float]) -> float:
    return sum(s.count * cost[s.name] for s in shards)


def instance_seeds(base_seed: int, first: int, count: int) -> list[int]:
    """Seeds of global instances [first, first + count): instance i's values come from its own
    generator seeded with (base_seed, i)."""
    return [(base_seed, first + i) for i in range(count)]
