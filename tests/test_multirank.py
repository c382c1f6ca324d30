"""The multi-GPU path on the CPU: two gloo ranks shard moduli the way `bench.py --gpus N`
does (no data-path collective), reduce time by max and records by sum, and gather the
per-modulus results -- which must equal the single-process results."""
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
    for j in range(6):
        M = W.draw_modulus(700 + j)
        Q = W.eligible_pool(M, 5518)
        k = rng.randint(8, 14)
        Qs = Q[: k + rng.randint(3, 20)]
        out.append((M, Qs, Qs[:k], rng.randint(1, 3), W.product(Qs[:k]) * 10 ** 6))
    return out


def _rank(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch
    import torch.distributed as dist

    import bench
    import oracle as O
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        sched = [w.name for w in bench.step_seeds(5, world, rank)]
        mine = _small()[rank::world]                       # this rank's moduli
        res = [(M, sorted((tuple(D), tuple(I)) for D, I in O.solve_exhaustive(M, Q, B0, r, B)[0]))
               for M, Q, B0, r, B in mine]
        t = torch.tensor([0.5 + rank], dtype=torch.float64)   # per-rank "device seconds"
        n = torch.tensor([1000.0 * (rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(n, op=dist.ReduceOp.SUM)
        g = [None] * world
        dist.all_gather_object(g, (sched, res))
        if rank == 0:
            out.put((float(t.item()), float(n.item()), g))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(600)
def test_two_gloo_ranks_shard_moduli():
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import bench
    import oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    tmax, nsum, gathered = q.get(timeout=500)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert tmax == 1.5 and nsum == 3000.0                 # max over ranks, sum over ranks
    s0, s1 = gathered[0][0], gathered[1][0]
    # every step gives each rank a different modulus; together they are the two-rank schedule
    assert len(s0) == len(s1) == 5 and all(a != b for a, b in zip(s0, s1))
    both = [w.name for w in bench.step_seeds(5, 2, 0)] + [w.name for w in bench.step_seeds(5, 2, 1)]
    assert sorted(both) == sorted(s0 + s1)
    # the sharded results are the single-process results
    sharded = {M: pairs for _, res in gathered for M, pairs in res}
    for M, Q, B0, r, B in _small():
        want = sorted((tuple(D), tuple(I)) for D, I in O.solve_exhaustive(M, Q, B0, r, B)[0])
        assert sharded[M] == want
