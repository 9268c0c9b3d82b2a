"""Sharding independent worlds and served jobs over the GPUs of a node.

Worlds never exchange data, so sharding needs no collective on the data path:
every rank computes the same assignment from the same inputs (the seeded
world list, or the job specs in arrival order) and steps only its own share,
one process and one CUDA device per rank.  The reference has no counterpart;
its analogue is the contiguous per-thread pair ranges of
`processPairsParallel` (src/narrow_phase.zig:1538-1632), with worlds in place
of pairs and a cost estimate in place of equal counts.

Cost estimates:
  * world_cost: one world step's device time grows about linearly with the
    bodies (pair count, contact points and the colour count all follow the
    body count in these scenes), plus a fixed per-world share of the batch
    launch; measured per-world times (VoxelWorldBatch.times) can be passed
    instead.
  * job_cost: a served job's world cost times its steps.
"""
from __future__ import annotations

import heapq


def world_cost(n_bodies: int) -> float:
    """Estimated relative cost of one step of a world of n_bodies bodies."""
    return 16.0 + float(n_bodies)


def job_cost(n_bodies: int, steps: int) -> float:
    """Estimated relative cost of a served job: steps x world_cost."""
    return float(steps) * world_cost(n_bodies)


def partition(costs, n_ranks: int) -> list:
    """Longest-processing-time-first partition of items with the given costs
    into n_ranks lists of item indices: items in decreasing cost (ties by
    index) go to the least-loaded rank (ties by rank).  Deterministic, so every
    rank computes the same partition.  Each list is in increasing index order.
    The largest load is at most 4/3 of the optimum (Graham's bound)."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be at least 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(n_ranks)]
    out = [[] for _ in range(n_ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(x) for x in out]


def assign_jobs(jobs, n_ranks: int, cost=None) -> list:
    """Rank of each job, decided in arrival order as a dispatcher would: a job
    goes to the rank with the least estimated work still outstanding at its
    arrival (each rank assumed to retire `rate` cost units per second,
    equal for all ranks, so only the order of loads matters), ties by rank.
    `jobs` holds dicts with arrival, bodies and steps; `cost` maps a job to
    its cost (job_cost by default)."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be at least 1")
    cost = cost or (lambda j: job_cost(j["bodies"], j["steps"]))
    # outstanding work per rank at the current arrival time: a rank's queue
    # drains at one cost unit per unit of drain time; the drain rate is set
    # so that the whole stream keeps every rank busy on average
    total = sum(cost(j) for j in jobs)
    span = max((j["arrival"] for j in jobs), default=0.0) or 1.0
    rate = total / span / n_ranks if total > 0 else 1.0
    backlog = [0.0] * n_ranks
    last = 0.0
    out = []
    for j in sorted(range(len(jobs)), key=lambda k: (jobs[k]["arrival"], k)):
        t = jobs[j]["arrival"]
        drained = (t - last) * rate
        backlog = [max(0.0, b - drained) for b in backlog]
        last = t
        r = min(range(n_ranks), key=lambda k: (backlog[k], k))
        backlog[r] += cost(jobs[j])
        out.append((j, r))
    ranks = [0] * len(jobs)
    for j, r in out:
        ranks[j] = r
    return ranks


def imbalance(costs, parts) -> float:
    """Largest rank load over the mean rank load (1.0 is perfect)."""
    loads = [sum(float(costs[i]) for i in p) for p in parts]
    mean = sum(loads) / len(loads) if loads else 0.0
    return max(loads) / mean if mean > 0 else 1.0
