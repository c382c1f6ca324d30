"""Serving loop host logic on the CPU: footprint upper bounds and admission."""
import itertools
import math
import random
import threading
import time
import types

import pytest

from carmichael_frontier_b200 import serve, workloads as W
from carmichael_frontier_b200.serve import Server, count_ge_upper, count_lt_upper


def test_count_bounds_are_upper_bounds():
    rng = random.Random(3)
    for _ in range(30):
        M = W.draw_modulus(rng.randrange(10 ** 6))
        P = W.eligible_pool(M, 10 ** 5)[: rng.randint(6, 22)]
        r = rng.randint(1, min(5, len(P)))
        prods = [math.prod(c) for c in itertools.combinations(P, r)]
        lo = rng.choice(prods)
        hi = rng.choice(prods)
        ge = sum(1 for x in prods if x >= lo)
        lt = sum(1 for x in prods if x < hi)
        ub_ge, ub_lt = count_ge_upper(P, r, lo), count_lt_upper(P, r, hi)
        assert ge <= ub_ge <= math.comb(len(P), r)
        assert lt <= ub_lt <= math.comb(len(P), r)


def _fake_server(budget, slots, log):
    active = []
    lock = threading.Lock()

    def solve(state, inst):
        with lock:
            active.append(inst)
            log.append(("start", inst.rid, [a.rid for a in active], sum(a.need for a in active)))
        time.sleep(inst.dt)
        with lock:
            active.remove(inst)
        return types.SimpleNamespace(hits=[], rid=inst.rid)

    return Server(slots=slots, budget=budget, solve_fn=solve).start()


def test_admission_respects_budget_and_runs_oversize_alone():
    rng = random.Random(1)
    log = []
    srv = _fake_server(budget=100, slots=4, log=log)
    reqs = [types.SimpleNamespace(rid=i, need=rng.choice([10, 30, 60, 150]), dt=rng.uniform(0.001, 0.01))
            for i in range(60)]
    ts = [srv.submit(q) for q in reqs]
    for t in ts:
        assert t.done.wait(20)
    srv.stop()
    assert all(t.error is None and t.result.rid == t.inst.rid for t in ts)
    for _tag, rid, running, used in log:
        need = reqs[rid].need
        if need > 100:
            assert running == [rid]            # larger than the budget: alone
        else:
            assert used <= 100 and len(running) <= 4
    assert max(len(e[2]) for e in log) > 1      # requests did overlap
    assert srv.adm.peak <= 100 and srv.adm.used == 0


def test_no_starvation_of_large_requests():
    log = []
    srv = _fake_server(budget=100, slots=4, log=log)
    big = types.SimpleNamespace(rid=0, need=90, dt=0.001)
    smalls = [types.SimpleNamespace(rid=i, need=20, dt=0.02) for i in range(1, 40)]
    ts = [srv.submit(smalls[0]), srv.submit(big)] + [srv.submit(q) for q in smalls[1:]]
    for t in ts:
        assert t.done.wait(30)
    srv.stop()
    order = [e[1] for e in log]
    assert order.index(0) <= srv.adm.max_bypass + 2


def test_poisson_stats_shape():
    srv = _fake_server(budget=1000, slots=2, log=[])
    reqs = [types.SimpleNamespace(rid=i, need=1, dt=0.002) for i in range(20)]
    st, ts = serve.run_poisson(srv, reqs, rate=500.0, seed=2)
    srv.stop()
    assert st["requests"] == 20 and st["errors"] == 0
    assert st["p50_ms"] <= st["p99_ms"] and st["throughput_rps"] > 0


def test_footprint_reports_work_and_the_priority_class_takes_the_fast_path():
    # the footprint's record estimate is at least the records the solve will touch, and the server
    # sends the chosen class (requests at or above large_work, those below, or neither) to the
    # worker's high-priority path
    import math

    from carmichael_frontier_b200 import serve, workloads as W
    from carmichael_frontier_b200.solve import Instance, Tuning
    insts = [Instance.build(w.M, w.Q, w.B0, w.r, w.B) for w in W.config5_requests(12)]
    for x in insts:
        fp = serve.footprint(x, Tuning(strategy="auto"))
        assert fp["work"] > 0
        if fp["strategy"] == "fused":
            assert fp["work"] == math.comb(len(x.B0), x.r) + math.comb(len(x.INS), x.r)
    seen = []

    class Job:
        def __init__(self, work):
            self.need, self.work = 1, work

    want = {"large": [(5, False), (7, False), (100, True), (5000, True)],
            "small": [(5, True), (7, True), (100, False), (5000, False)],
            "none": [(5, False), (7, False), (100, False), (5000, False)]}
    for prio, expect in want.items():
        seen = []
        srv = serve.Server(slots=2, budget=10, solve_fn=lambda st, inst: None, large_work=100, priority=prio)
        orig = srv._solve
        srv._solve = lambda state, inst, fast=False, orig=orig, seen=seen: seen.append((inst.work, fast)) or \
            orig(state, inst, fast)
        srv.start()
        for w in (5, 100, 7, 5000):
            srv.submit(Job(w)).done.wait()
        srv.stop()
        assert sorted(seen) == expect, prio
    with pytest.raises(ValueError):
        serve.Server(slots=1, budget=10, solve_fn=lambda st, inst: None, priority="fastest")


def test_large_requests_run_one_at_a_time_in_order():
    # requests at or above large_work share a one-request lane in arrival order; small ones run
    # beside a large one and pass a large one that waits for the lane
    active, log = [], []
    lock = threading.Lock()

    def solve(state, inst):
        with lock:
            active.append(inst)
            log.append((inst.rid, [a.rid for a in active if a.work >= 100]))
        time.sleep(inst.dt)
        with lock:
            active.remove(inst)
        return types.SimpleNamespace(hits=[], rid=inst.rid)

    srv = Server(slots=4, budget=1000, solve_fn=solve, large_work=100).start()
    big = [types.SimpleNamespace(rid=i, need=1, work=500, dt=0.03) for i in range(3)]
    small = [types.SimpleNamespace(rid=10 + i, need=1, work=5, dt=0.002) for i in range(12)]
    ts = [srv.submit(q) for q in (big[0], big[1], small[0], big[2], *small[1:])]
    for t in ts:
        assert t.done.wait(20)
    srv.stop()
    assert all(len(larges) <= 1 for _rid, larges in log)
    starts = [rid for rid, _ in log]
    assert [r for r in starts if r < 10] == [0, 1, 2]
    assert starts.index(10) < starts.index(1)                 # a small one passed the waiting large one
    assert srv.adm.large_running == 0 and srv.adm.used == 0


def test_small_requests_beside_a_large_one_are_capped():
    active, log = [], []
    lock = threading.Lock()

    def solve(state, inst):
        with lock:
            active.append(inst)
            log.append((inst.rid, sum(1 for a in active if a.work >= 100), sum(1 for a in active if a.work < 100)))
        time.sleep(inst.dt)
        with lock:
            active.remove(inst)
        return types.SimpleNamespace(hits=[], rid=inst.rid)

    srv = Server(slots=4, budget=1000, solve_fn=solve, large_work=100, beside_large=1).start()
    big = types.SimpleNamespace(rid=0, need=1, work=500, dt=0.05)
    small = [types.SimpleNamespace(rid=1 + i, need=1, work=5, dt=0.005) for i in range(10)]
    ts = [srv.submit(big)] + [srv.submit(q) for q in small]
    for t in ts:
        assert t.done.wait(20)
    srv.stop()
    assert all(nsmall <= 1 for _rid, nlarge, nsmall in log if nlarge)
    assert any(nlarge and nsmall for _rid, nlarge, nsmall in log)    # one small ran beside the large one
