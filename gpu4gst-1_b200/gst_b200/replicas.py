"""Multi-GPU query sharding: one process per GPU, graph replicated per GPU.

Queries are independent, so the multi-GPU form of the solve is replicas:
every rank holds the whole graph and groups, takes a disjoint share of the
queries, and only the (tiny) per-query results travel between ranks.  There is
no collective on the data path; torch.distributed (NCCL on GPUs, gloo on CPU)
is used for barriers, the max-over-ranks timer and gathering results.

Shares are balanced by an estimate of each query's work (table size
V x 2^k x (D+1), the quantity admission is bounded by) with a greedy
longest-first assignment, which keeps mixed k / D batches even across ranks.
"""
from __future__ import annotations

import numpy as np


def query_weight(k: int, D: int) -> float:
    """Relative work of a query: table entries per vertex."""
    return float((1 << k) * (1 if D < 0 else D + 1))


def shard(queries, Ds, world: int) -> list:
    """Splits query indices into `world` shares of near-equal estimated work.
    Deterministic: every rank computes the same split."""
    n = len(queries)
    w = np.array([query_weight(len(set(int(x) for x in q)), -1 if Ds is None else int(Ds[i]))
                  for i, q in enumerate(queries)], dtype=np.float64)
    order = sorted(range(n), key=lambda i: (-w[i], i))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda j: (load[j], j))
        parts[r].append(i)
        load[r] += w[i]
    return [sorted(p) for p in parts]


def solve_sharded(solve_batch, queries, Ds=None, group=None):
    """Solves `queries` across the ranks of `group` (torch.distributed).

    solve_batch(list_of_queries, list_of_D) -> list of results with a `.cost`
    attribute (the engine's Engine.solve_batch, or any stand-in).  Returns,
    on every rank, the list of (cost, feasible) in query order.
    """
    import torch.distributed as dist

    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    parts = shard(queries, Ds, world)
    mine = parts[rank]
    res = solve_batch([queries[i] for i in mine], None if Ds is None else [Ds[i] for i in mine]) if mine else []
    local = [(i, int(r.cost), bool(r.feasible)) for i, r in zip(mine, res)]
    if world == 1:
        gathered = [local]
    else:
        gathered = [None] * world
        dist.all_gather_object(gathered, local, group=group)
    out = [None] * len(queries)
    for part in gathered:
        for i, c, f in part:
            out[i] = (c, f)
    return out
