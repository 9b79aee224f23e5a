"""Multi-GPU batch partitioning: independent graphs sharded across ranks.

A single graph does not shard (matching, contraction and refinement need whole
neighbourhoods at every level), but a batch of independent graphs does: each rank
(one process per GPU) partitions its share with the batched C-ABI call
(``hp_partition_batch``) on its own device, and the per-graph results are gathered
on the host.  There is no collective on the data path; the only exchange is the
final gather of the part arrays (``all_gather_object`` over the process group).

The share of each rank is a greedy longest-processing-time assignment on the
per-graph cost ``m + n``: graphs in decreasing cost order (ties by index) go to the
least-loaded rank (ties by rank number).  The assignment is a pure function of the
graph sizes and the world size, so every rank computes the same one without
communication.
"""
from __future__ import annotations

import heapq
from typing import Callable, Sequence

import numpy as np


def graph_cost(g) -> int:
    """Work estimate of one graph: directed adjacency entries plus vertices."""
    return int(g.nedges) + int(g.nvtxs)


def assign_lpt(costs: Sequence[int], world: int) -> list[list[int]]:
    """Greedy LPT assignment of items (by cost) to ``world`` ranks.

    Returns one ascending list of item indices per rank; every item appears in
    exactly one list."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-int(costs[i]), i))
    heap = [(0, r) for r in range(world)]
    shares: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + int(costs[i]), r))
    return [sorted(s) for s in shares]


BatchFn = Callable[[list, list, float, object], tuple]


def partition_batch_sharded(graphs: Sequence, nparts, ubfactor: float = 1.03, options=None, *,
                            group=None, batch_fn: BatchFn | None = None, ctx=None):
    """Partition ``graphs`` across the ranks of ``group`` (torch.distributed).

    Each rank partitions its LPT share with ``batch_fn(graphs, ks, ubfactor, options)``
    (default: ``ctx.partition_batch`` of a :class:`hunyuansc25_b200.Context` on this
    rank's device), then the results are all-gathered so that every rank returns the
    full ``(parts, cuts)`` in input order.  Each graph's result is the same as a
    single-graph call on it, whatever the world size.

    Returns ``(parts, cuts, share)`` where ``share`` lists the indices this rank ran.
    """
    import torch.distributed as dist

    G = len(graphs)
    ks = [int(k) for k in np.broadcast_to(np.asarray(nparts), (G,))]
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    shares = assign_lpt([graph_cost(g) for g in graphs], world)
    mine = shares[rank]
    if batch_fn is None:
        if ctx is None:
            raise ValueError("partition_batch_sharded needs ctx (a Context) or batch_fn")

        def batch_fn(gs, kk, ub, opt):
            return ctx.partition_batch(gs, kk, ub, opt)

    if mine:
        p, c = batch_fn([graphs[i] for i in mine], [ks[i] for i in mine], ubfactor, options)
        local = [(i, np.asarray(p[j], np.int32), int(c[j])) for j, i in enumerate(mine)]
    else:
        local = []
    if world > 1:
        gathered: list = [None] * world
        dist.all_gather_object(gathered, local, group=group)
    else:
        gathered = [local]
    parts: list = [None] * G
    cuts = np.zeros(G, np.int64)
    for chunk in gathered:
        for i, p, c in chunk:
            parts[i] = p
            cuts[i] = c
    missing = [i for i in range(G) if parts[i] is None]
    if missing:
        raise RuntimeError(f"sharded batch lost graphs {missing[:8]}")
    return parts, cuts, mine
