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

One modulus too large for one GPU's time splits the other way (the I-rank range; the D table is
built on every rank, it is the small side):

  windows(n_I, world)           contiguous I-rank windows of near-equal size, one per rank
  run_split(solve_window, n_I, group)
                                this rank joins its window with solve_window(lo, hi) -> SolveResult,
                                and every rank gets the merged result: the whole instance's pairs and
                                hits, as one solve over all I ranks gives them
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


def windows(n: int, world: int) -> list[tuple[int, int]]:
    """[lo, hi) I-rank windows covering [0, n), one per rank, sizes differing by at most one."""
    if world < 1:
        raise ValueError("world must be at least 1")
    q, rem = divmod(int(n), world)
    out, lo = [], 0
    for r in range(world):
        hi = lo + q + (1 if r < rem else 0)
        out.append((lo, hi))
        lo = hi
    return out


def merge_windows(parts: list):
    """One SolveResult from the SolveResults of disjoint I-rank windows of one instance: counts
    added, pairs and hits merged in the order a single solve reports them."""
    from .solve import SolveResult
    parts = [p for p in parts if p is not None]
    if not parts:
        raise ValueError("no window results to merge")
    hits = sorted((h for p in parts for h in p.hits), key=lambda h: (h.n, h.D, h.I))
    pairs = sorted(x for p in parts for x in p.pairs)
    first = parts[0]
    return SolveResult(hits=hits, n_D=first.n_D, n_I=sum(p.n_I for p in parts),
                       residue_pairs=sum(p.residue_pairs for p in parts), screened=sum(p.screened for p in parts),
                       above_bound=sum(p.above_bound for p in parts), rejected=sum(p.rejected for p in parts),
                       plan=dict(first.plan), pairs=pairs, launches=sum(p.launches for p in parts))


def run_split(solve_window, n_I: int, group=None):
    """Join this rank's I-rank window of one instance and gather the whole result.

    solve_window(lo, hi) -> SolveResult of the I ranks [lo, hi) (the D side complete).  With no
    process group (or world size 1) the whole range is joined here.  Returns (merged SolveResult,
    this rank's window)."""
    import torch.distributed as dist
    if group is None and not (dist.is_available() and dist.is_initialized()):
        world, rank = 1, 0
    else:
        world, rank = dist.get_world_size(group), dist.get_rank(group)
    win = windows(n_I, world)[rank]
    mine = solve_window(*win)
    if world == 1:
        return mine, win
    gathered: list = [None] * world
    dist.all_gather_object(gathered, mine, group=group)
    return merge_windows(gathered), win
