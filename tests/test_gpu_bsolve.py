"""The product-bounded solve (filtered producers + record hash join) against the
exhaustive oracle, the unpruned fused join and the reference's positive control."""
import math
import random

import pytest

import oracle as O
from carmichael_frontier_b200 import Solver, Tuning, workloads as W
from carmichael_frontier_b200.bounded import BoundedGenerator
from carmichael_frontier_b200.solve import Instance

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bounded(cuda):
    return Solver(cuda, tuning=Tuning(strategy="bounded"))


@pytest.fixture(scope="module")
def fused(cuda):
    return Solver(cuda, tuning=Tuning(strategy="fused"))


def hits_of(res):
    return [(h.D, h.I, h.n) for h in res.hits]


@pytest.mark.parametrize("seed", range(6))
def test_bounded_small_vs_exhaustive(bounded, seed):
    rng = random.Random(70 + seed)
    M = W.draw_modulus(300 + seed)
    Q = W.eligible_pool(M, 5518)
    k = rng.randint(8, 20)
    r = rng.randint(1, 4)
    Qs = Q[: k + rng.randint(r, 40)]
    B0 = Qs[:k]
    P0 = W.product(B0)
    for B in (P0 * 10 ** rng.randint(0, 6), P0 * 10 ** 30, P0 // 10 ** 3 + 1):
        res = bounded.solve(M, Qs, B0, r, B)
        pairs, hits = O.solve_exhaustive(M, Qs, B0, r, B)
        assert hits_of(res) == [(tuple(D), tuple(I), n) for D, I, n in hits]
        assert res.rejected == 0
        # every pair the join reports is an equal-residue pair, and every pair of a hit is reported
        allp = {(tuple(D), tuple(I)) for D, I in pairs}
        assert set(res.pairs) <= allp
        assert {(h.D, h.I) for h in res.hits} <= set(res.pairs)


def test_bounded_equals_fused_on_serving_requests(bounded, fused):
    # requests of the serving stream (k = 64..100, B = prod(B0) * 10^4): same hits either way
    for w in W.config5_requests(40):
        inst = Instance.build(w.M, w.Q, w.B0, w.r, w.B)
        if math.comb(len(inst.INS), inst.r) > 3 * 10 ** 8 or math.comb(len(inst.B0), inst.r) > 3 * 10 ** 8:
            continue
        a = bounded.solve_instance(inst)
        b = fused.solve_instance(inst)
        assert a.plan["strategy"] == "bounded"
        assert hits_of(a) == hits_of(b) and a.rejected == 0
        assert a.n_I <= b.n_I and a.n_D <= b.n_D


def test_positive_control_sides_and_hit(cuda, golden, bounded):
    # the reference's own filtered sides at M0, r = 7: 2,013,093 I and 37,332,675 D records
    pc = golden["positive_control"]
    g = BoundedGenerator(cuda)
    P0 = O.product(pc["B0"])
    total = sum(int(k.numel()) for k, _ in g.generate_I(pc["INS"], pc["r"], pc["M"], P0, int(pc["Icap"])))
    assert total == pc["i_records"]
    _, _, nd = g.generate_D(pc["B0"], pc["r"], pc["M"], int(pc["Dmin"]))
    assert nd == pc["d_records"]
    N = int(pc["N"])
    res = bounded.solve(pc["M"], pc["B0"] + pc["INS"], pc["B0"], pc["r"], N)
    assert [(list(h.D), list(h.I), str(h.n)) for h in res.hits] == [tuple(p) for p in pc["pairs"]]
