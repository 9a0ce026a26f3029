"""Partitioning one batched sweep across ranks (one process per GPU).

A sweep is a set of independent trap instances; no instance exchanges data
with another during a step, so the sweep shards by instance with no per-step
collective. Each rank runs its share of the SAME instance list; at the end a
single host gather brings the per-instance results back to rank 0 in
instance order.

Cost model (per step, arbitrary units): an all-pairs instance of N particles
costs N (N - 1) pair interactions; a tree-solver instance (FMM, Barnes-Hut)
costs about N log2 N times 4,000 pair interactions (measured on one B200: a
1,048,576-particle FMM evaluation at p = 4 takes 33 ms, the time of
6.6e10 all-pairs interactions at 5e-13 s each); a cutoff instance costs N.

The assignment is LPT (longest processing time first): instances sorted by
descending cost (ties by index) go one at a time to the least-loaded rank
(ties to the lowest rank). Graham's bound holds: the largest load is at most
4/3 - 1/(3 R) of the optimum, and at most the mean load plus the largest
single cost.
"""
from __future__ import annotations

import math
from typing import Iterable, Sequence

# method codes of amk_batch_set / amk_batch_autotune
METHOD_CUTOFF, METHOD_BARNES_HUT, METHOD_FMM, METHOD_ALLPAIRS = 0, 1, 2, 3

TREE_COST_PER_NLOGN = 4000.0  # relative to one all-pairs pair interaction


def instance_cost(n: int, method) -> float:
    """Per-step cost estimate of one instance of `n` particles."""
    n = max(int(n), 0)
    if isinstance(method, str):
        method = {"allpairs": METHOD_ALLPAIRS, "fast-multipole": METHOD_FMM, "fmm": METHOD_FMM,
                  "barnes-hut": METHOD_BARNES_HUT, "standard": METHOD_CUTOFF,
                  "cutoff": METHOD_CUTOFF}.get(method, METHOD_ALLPAIRS)
    if method == METHOD_ALLPAIRS:
        return float(n) * max(n - 1, 0)
    if method in (METHOD_FMM, METHOD_BARNES_HUT):
        return TREE_COST_PER_NLOGN * n * math.log2(max(n, 2))
    return float(n)


def partition_lpt(costs: Sequence[float], world: int) -> list[list[int]]:
    """Instance indices per rank (each list ascending). Deterministic: every
    rank computes the same assignment from the same costs."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


def loads(costs: Sequence[float], parts: Iterable[Iterable[int]]) -> list[float]:
    return [sum(float(costs[i]) for i in p) for p in parts]


def imbalance(costs: Sequence[float], parts: Sequence[Sequence[int]]) -> float:
    """Largest rank load over the mean load (1.0 = perfect balance)."""
    ld = loads(costs, parts)
    mean = sum(ld) / max(len(ld), 1)
    return max(ld) / mean if mean > 0 else 1.0


def gather_instance_rows(local_ids: Sequence[int], local_rows: Sequence, n_instances: int,
                         world: int, rank: int):
    """Gathers per-instance rows (any picklable values) from every rank to
    rank 0 through torch.distributed (gloo or NCCL process group already
    initialised when world > 1). Returns the rows in instance order on rank 0
    and None elsewhere. Every instance must be reported by exactly one rank."""
    if len(local_ids) != len(local_rows):
        raise ValueError("one row per local instance")
    mine = list(zip((int(i) for i in local_ids), local_rows))
    if world == 1:
        everything = [mine]
    else:
        import torch.distributed as dist
        everything = [None] * world
        dist.all_gather_object(everything, mine)
    if rank != 0:
        return None
    out = [None] * n_instances
    seen = [False] * n_instances
    for part in everything:
        for i, row in part:
            if not 0 <= i < n_instances or seen[i]:
                raise ValueError(f"instance {i} reported twice or out of range")
            seen[i] = True
            out[i] = row
    missing = [i for i, s in enumerate(seen) if not s]
    if missing:
        raise ValueError(f"instances never reported: {missing[:8]}")
    return out
