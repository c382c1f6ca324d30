"""Serving loop on the GPU: every result is the same alone and in the mix."""
import math

import pytest

from carmichael_frontier_b200 import Solver, Tuning, serve, workloads as W
from carmichael_frontier_b200.solve import Instance

pytestmark = pytest.mark.gpu


def summary(res):
    return (res.n_D, res.n_I, res.residue_pairs, res.above_bound, res.rejected, sorted(res.pairs),
            [(h.D, h.I, h.n) for h in res.hits])


def requests(count, limit=2 * 10 ** 8):
    out = []
    for w in W.config5_requests(count * 3):
        inst = Instance.build(w.M, w.Q, w.B0, w.r, w.B)
        if math.comb(len(inst.INS), inst.r) <= limit:
            out.append(inst)
        if len(out) == count:
            break
    return out


def test_results_same_alone_and_in_the_mix(cuda):
    insts = requests(24)
    alone = Solver(cuda, tuning=Tuning(strategy="auto", max_nodes=1 << 22))
    ref = [summary(alone.solve_instance(x)) for x in insts]
    srv = serve.Server(cuda, slots=4, strategy="auto").start()
    ts = [srv.submit(x) for x in insts]
    for t in ts:
        assert t.done.wait(600)
    srv.stop()
    assert all(t.error is None for t in ts), [t.error for t in ts if t.error]
    assert [summary(t.result) for t in ts] == ref
    assert srv.adm.peak <= srv.adm.budget


def test_bounded_frontier_blocks_and_plain_form_agree(cuda):
    insts = requests(6)
    small = Solver(cuda, tuning=Tuning(strategy="bounded", max_nodes=2000))
    big = Solver(cuda, tuning=Tuning(strategy="bounded"))
    fused = Solver(cuda, tuning=Tuning(strategy="fused"))
    for x in insts:
        a, b, c = small.solve_instance(x), big.solve_instance(x), fused.solve_instance(x)
        p = serve.plain_solve(x, device=cuda)
        assert summary(a) == summary(b)
        assert [(h.D, h.I, h.n) for h in a.hits] == [(h.D, h.I, h.n) for h in c.hits]
        assert (p.n_D, p.n_I, sorted(p.pairs), [h.n for h in p.hits]) == (a.n_D, a.n_I, sorted(a.pairs),
                                                                          [h.n for h in a.hits])


def test_poisson_run_reports_latency(cuda):
    insts = requests(12)
    srv = serve.Server(cuda, slots=3, strategy="auto").start()
    st, ts = serve.run_poisson(srv, insts, rate=50.0, seed=1)
    srv.stop()
    assert st["requests"] == 12 and st["errors"] == 0
    assert 0 < st["p50_ms"] <= st["p99_ms"]
