"""Moduli sharded over ranks: one process per GPU, no data-path collective.

Moduli are independent instances, so a portfolio, a census family or a request stream splits across
ranks by modulus (the reference's campaigns split the same way across machines with FAM_SHARD=i/n,
gpu/run_mstar_family.py:47-48).  Each rank solves its share on its own GPU; the only collectives are
the gather of the (small) per-modulus results and the max-over-ranks of the device time.

  assign(weights, world)        balanced shares: longest-processing-time order, each instance to the
                                rank with the least work so far (deterministic, every rank computes
                                the same assignment without communicating)
  run_sharded(items, weights, solve_share, group)
                                this rank solves its share with solve_share(list of items) and gets
                                back every rank's results, in the input order
"""
from __future__ import annotations

import heapq


def assign(weights, world: int) -> list[list[int]]:
    """Indices of the items each rank takes, each list in input order."""
    if world < 1:
        raise ValueError("world must be at least 1")
    order = sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i))
    heap = [(0.0, r) for r in range(world)]
    shares: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + float(weights[i]), r))
    return [sorted(s) for s in shares]


def run_sharded(items, weights, solve_share, group=None) -> tuple[list, list[int]]:
    """Solve this rank's share of `items` and gather every rank's results.

    solve_share(list of items) -> list of results, one per item, in that order.  With no process
    group (or world size 1) everything is solved here.  Returns (results in input order, the indices
    this rank solved)."""
    import torch.distributed as dist
    if group is None and not (dist.is_available() and dist.is_initialized()):
        world, rank = 1, 0
    else:
        world, rank = dist.get_world_size(group), dist.get_rank(group)
    shares = assign(weights, world)
    mine = shares[rank]
    got = solve_share([items[i] for i in mine])
    if len(got) != len(mine):
        raise RuntimeError("solve_share returned a different number of results than items")
    if world == 1:
        return list(got), mine
    gathered: list = [None] * world
    dist.all_gather_object(gathered, (rank, list(got)), group=group)
    out: list = [None] * len(items)
    for r, res in gathered:
        for i, x in zip(shares[r], res):
            out[i] = x
    return out, mine
