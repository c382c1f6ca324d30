"""The one-call bounded join (cf_bounded_join) against the level loop and the oracle, on the GPU.

BoundedSolve runs an instance through cf_bounded_join when it can (modulus below 2^64, caps below
2^128) and through its Python level loop otherwise; both must give the same pairs and side sizes,
and the exhaustive oracle the same pairs on small instances."""
import math
import random

import pytest

import oracle as O
from carmichael_frontier_b200 import bsolve, driver, workloads as W
from carmichael_frontier_b200.solve import Solver, Tuning

pytestmark = pytest.mark.gpu


def _both(cuda, B0, INS, r, M, P0, Icap, Dmin, split, hmax):
    s = Solver(cuda, tuning=Tuning(strategy="bounded"))
    bs = bsolve.BoundedSolve(s)
    got_native = bs.join(B0, INS, r, M, P0, Icap, Dmin, split, hmax)
    bs.native = False
    got_loop = bs.join(B0, INS, r, M, P0, Icap, Dmin, split, hmax)
    return got_native, got_loop


@pytest.mark.parametrize("seed", range(4))
def test_one_call_join_equals_level_loop(cuda, seed):
    rng = random.Random(77 + seed)
    for j in range(5):
        M = W.draw_modulus(5000 + 17 * seed + j)
        Q = W.eligible_pool(M, 20_000)
        k = rng.randint(20, 64)
        r = rng.randint(1, 6)
        B0, INS = Q[:k], Q[k:k + rng.randint(r + 2, 150)]
        if len(INS) < r:
            continue
        P0 = math.prod(B0)
        U = P0 * rng.choice([10 ** 3, 10 ** 8, 10 ** 15])
        Icap, Dmin, _cap_r, aff = driver.instance_bounds(B0, INS, r, U)
        if len(aff) < r:
            continue
        split = aff[rng.randrange(len(aff))] if rng.random() < 0.5 else None
        hmax = rng.randint(0, r) if split is not None else None
        (pn, dn, inn, plan), (pl, dl, il, _) = _both(cuda, B0, aff, r, M, P0, Icap, Dmin, split, hmax)
        assert plan.get("native") and (dn, inn) == (dl, il)
        assert sorted(pn) == sorted(pl)


def test_one_call_join_against_the_oracle(cuda):
    rng = random.Random(3)
    for j in range(6):
        M = W.draw_modulus(6100 + j)
        Q = W.eligible_pool(M, 3000)[:36]
        B0, r = Q[:12], 2 + j % 3
        P0 = math.prod(B0)
        B = P0 * 10 ** 7
        pairs, _hits = O.solve_exhaustive(M, Q, B0, r, B)
        from carmichael_frontier_b200.solve import Instance
        inst = Instance.build(M, Q, B0, r, B)
        Icap, Dmin = bsolve.caps(inst)
        s = Solver(cuda, tuning=Tuning(strategy="bounded"))
        bs = bsolve.BoundedSolve(s)
        got, nD, nI, plan = bs.join(inst.B0, inst.INS, r, M, P0, Icap, Dmin)
        assert plan.get("native")
        want = {(D, I) for D, I in ((tuple(D), tuple(I)) for D, I in pairs)
                if math.prod(I) < Icap and math.prod(D) >= Dmin}
        assert {(tuple(inst.B0[x] for x in d), tuple(inst.INS[x] for x in i)) for d, i in got} == want
        bs.native = False                       # the level loop (its D table also under key forms)
        got2, _nD, _nI, plan2 = bs.join(inst.B0, inst.INS, r, M, P0, Icap, Dmin)
        assert not plan2.get("native")
        assert {(tuple(inst.B0[x] for x in d), tuple(inst.INS[x] for x in i)) for d, i in got2} == want
