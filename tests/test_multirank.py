"""The multi-GPU path on the CPU: two gloo ranks run the product's sharding code.

carmichael_frontier_b200.shard assigns moduli to ranks and gathers the per-modulus results (the
only collectives besides the max-over-ranks of the device time); bench.py's step schedule gives each
rank its own moduli.  Here each rank solves its share with the CPU oracle in place of its GPU (the
only part that needs a device), and the gathered results must equal a single-process run, in input
order, with every modulus solved exactly once.  One instance split over the ranks by I-rank window
(shard.run_split, every rank with the whole D side) must give the whole instance's pair set."""
import datetime
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _small():
    import random

    from carmichael_frontier_b200 import workloads as W
    rng = random.Random(5)
    out = []
    for j in range(7):
        M = W.draw_modulus(700 + j)
        Q = W.eligible_pool(M, 5518)
        k = rng.randint(8, 14)
        Qs = Q[: k + rng.randint(3, 20)]
        out.append((M, Qs, Qs[:k], rng.randint(1, 3), W.product(Qs[:k]) * 10 ** 6))
    return out


def _solve_on_this_rank(items):
    import oracle as O
    return [sorted((tuple(D), tuple(I)) for D, I in O.solve_exhaustive(M, Q, B0, r, B)[0])
            for M, Q, B0, r, B in items]


def _window_solve(item, lo, hi):
    """The join of one instance over its I ranks [lo, hi), by brute force on the CPU (lexicographic
    ranks: itertools.combinations order), as a SolveResult like the GPU solve's."""
    import itertools
    import math

    from carmichael_frontier_b200.solve import SolveResult
    M, Q, B0, r, B = item
    B0 = sorted(B0)
    INS = sorted(set(Q) - set(B0))
    P0 = math.prod(B0)
    byres: dict = {}
    for D in itertools.combinations(B0, r):
        byres.setdefault(math.prod(D) % M, []).append(D)
    pairs = []
    for i, I in enumerate(itertools.combinations(INS, r)):
        if i >= hi:
            break
        if i >= lo:
            pairs += [(D, I) for D in byres.get(P0 * math.prod(I) % M, [])]
    return SolveResult(hits=[], n_D=math.comb(len(B0), r), n_I=hi - lo, residue_pairs=len(pairs), screened=0,
                       above_bound=0, rejected=0, pairs=sorted(pairs))


def _weights(items):
    import math
    return [math.comb(len(B0), r) + math.comb(len(Q) - len(B0), r) for _, Q, B0, r, _ in items]


def _rank(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch
    import torch.distributed as dist

    import bench
    from carmichael_frontier_b200 import shard
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        sched = [w.name for w in bench.step_seeds(5, world, rank)]
        items = _small()
        res, mine = shard.run_sharded(items, _weights(items), _solve_on_this_rank)
        t = torch.tensor([0.5 + rank], dtype=torch.float64)   # per-rank "device seconds"
        n = torch.tensor([1000.0 * (rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(n, op=dist.ReduceOp.SUM)
        g = [None] * world
        dist.all_gather_object(g, (sched, mine))
        # one instance split over the ranks by I-rank window (the D side on every rank)
        import math
        splits = []
        for item in items[:3]:
            nI = math.comb(len(item[1]) - len(item[2]), item[3])
            merged, win = shard.run_split(lambda lo, hi, item=item: _window_solve(item, lo, hi), nI)
            splits.append((merged.pairs, merged.n_I, merged.residue_pairs, win))
        out.put((rank, float(t.item()), float(n.item()), g, res, splits))
    finally:
        dist.destroy_process_group()


def test_windows_cover_the_rank_range_once():
    import sys
    sys.path.insert(0, ROOT)
    from carmichael_frontier_b200 import shard
    for n in (0, 1, 7, 100, 12345):
        for world in (1, 2, 3, 8):
            w = shard.windows(n, world)
            assert len(w) == world and w[0][0] == 0 and w[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(w, w[1:]))
            assert max(hi - lo for lo, hi in w) - min(hi - lo for lo, hi in w) <= 1


def test_assignment_is_balanced_and_covers_every_item_once():
    import sys
    sys.path.insert(0, ROOT)
    from carmichael_frontier_b200 import shard
    w = [5, 1, 1, 1, 1, 1, 3, 2, 8, 1]
    for world in (1, 2, 3, 4, 16):
        sh = shard.assign(w, world)
        assert sorted(i for s in sh for i in s) == list(range(len(w)))
        loads = [sum(w[i] for i in s) for s in sh]
        assert max(loads) - min(loads) <= max(w)
        assert sh == shard.assign(w, world)                 # every rank computes the same shares


@pytest.mark.timeout(600)
def test_two_gloo_ranks_shard_moduli():
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import bench
    from carmichael_frontier_b200 import shard
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=500) for _ in range(2))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    items = _small()
    want = _solve_on_this_rank(items)                     # one process, every modulus
    import math
    for rank, tmax, nsum, gathered, res, splits in got:
        for item, (pairs, n_i, npairs, win) in zip(items[:3], splits):
            whole = _window_solve(item, 0, math.comb(len(item[1]) - len(item[2]), item[3]))
            assert pairs == whole.pairs and n_i == whole.n_I and npairs == whole.residue_pairs
            assert win == shard.windows(whole.n_I, 2)[rank]
        assert tmax == 1.5 and nsum == 3000.0             # max over ranks, sum over ranks
        assert res == want                                # every rank holds all results, in input order
        s0, s1 = gathered[0][0], gathered[1][0]
        # every step gives each rank a different modulus; together they are the two-rank schedule
        assert len(s0) == len(s1) == 5 and all(a != b for a, b in zip(s0, s1))
        both = [w.name for w in bench.step_seeds(5, 2, 0)] + [w.name for w in bench.step_seeds(5, 2, 1)]
        assert sorted(both) == sorted(s0 + s1)
        m0, m1 = gathered[0][1], gathered[1][1]           # each modulus solved by exactly one rank
        assert sorted(m0 + m1) == list(range(len(items))) and not set(m0) & set(m1)
        assert (m0, m1) == tuple(shard.assign(_weights(items), 2))
