"""The large-radius instance (seeded modulus, pool of 160 primes, r = 7) against the reference.

The whole instance (6.2e8 D x 1.19e10 I records) is beyond the reference's CPU engines, so the
reference pins a product-bounded sub-instance of it: every D record (Dmin = 0) against the I subsets
with prod(I) < Icap, about 2e8 records, produced by src/mitm64_ddump.cpp and
src/mitm64_idump_stream2.cpp and joined in numpy (tests/golden/make_golden.py --config4, the method of
gpu/validate_mitm_gpu2_pos.py:23-33).  Here:
  * the bounded producers give the same two record sets (counts and digests);
  * the fused join of the WHOLE instance, restricted to prod(I) < Icap, gives exactly the reference's
    pairs;
  * the streamed join of the two bounded sides, spilled to pinned host memory by residue range, gives
    the same pairs;
  * the bounded solve (record table of D probed by the I leaves) gives the same pairs.
"""
import math

import pytest

import oracle as O
from carmichael_frontier_b200 import bounded, bsolve, workloads as W
from carmichael_frontier_b200.solve import Instance, Solver, Tuning
from carmichael_frontier_b200.streamed import StreamedJoin
from carmichael_frontier_b200.tables import unrank_colex
from test_gpu_kat_large import dev_digest_add

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c4(golden):
    return golden["config4_bounded"]


def _want(c4):
    return sorted((tuple(d), tuple(i)) for d, i in c4["pairs"])


def test_instance_is_the_large_radius_config(c4):
    w = W.config4(0)
    assert (w.M, w.r, list(w.B0), list(w.INS)) == (c4["M"], c4["r"], c4["B0"], c4["INS"])
    assert len(c4["INS"]) == 96 and c4["d_records"] == math.comb(64, 7) and len(c4["pairs"]) > 0


def test_bounded_producers_match_reference_dumpers(cuda, c4):
    g = bounded.BoundedGenerator(cuda)
    P0 = O.product(c4["B0"])
    acc, n = (0, 0, 0), 0
    for k, i in g.generate_I(c4["INS"], c4["r"], c4["M"], P0, int(c4["Icap"]), max_records=1 << 27):
        acc = dev_digest_add(acc, k, i)
        n += k.numel()
    assert n == c4["i_records"] and O.record_digest_hex(acc) == c4["i_digest"]
    dk, di, nd = g.generate_D(c4["B0"], c4["r"], c4["M"], 0)
    assert nd == c4["d_records"]
    assert O.record_digest_hex(dev_digest_add((0, 0, 0), dk, di)) == c4["d_digest"]


def test_fused_whole_instance_restricted_to_the_bound(cuda, c4):
    w = W.config4(0)
    inst = Instance.build(w.M, w.Q, w.B0, w.r, w.B)
    res = Solver(cuda, tuning=Tuning(strategy="fused")).solve_instance(inst)
    Icap = int(c4["Icap"])
    got = sorted((tuple(D), tuple(I)) for D, I in res.pairs if math.prod(I) < Icap)
    assert got == _want(c4)
    assert res.residue_pairs >= len(got)


def test_streamed_join_of_the_bounded_sides(cuda, c4):
    g = bounded.BoundedGenerator(cuda)
    r, M, B0, INS = c4["r"], c4["M"], c4["B0"], c4["INS"]
    P0 = O.product(B0)
    sj = StreamedJoin(cuda, pbits=8)
    D = sj.spill_records(lambda: iter([g.generate_D(B0, r, M, 0, bitmask=2)[:2]]), M)
    I = sj.spill_records(lambda: g.generate_I(INS, r, M, P0, int(c4["Icap"]), max_records=1 << 26), M,
                         cap=1 << 26)
    assert (D.n, I.n) == (c4["d_records"], c4["i_records"])
    cand = sj.join(D, I)
    dids, iids = D.ids_np(), I.ids_np()
    got = sorted((tuple(B0[x] for x in unrank_colex(int(dids[int(a)]), r, len(B0))),
                  tuple(INS[x] for x in unrank_colex(int(iids[int(b)]), r, len(INS)))) for a, b in cand)
    assert got == _want(c4)


def test_bounded_solve_of_the_sub_instance(cuda, c4):
    s = Solver(cuda, tuning=Tuning(strategy="bounded"))
    bs = bsolve.BoundedSolve(s)
    r, B0, INS = c4["r"], c4["B0"], c4["INS"]
    pairs, nD, nI, _plan = bs.join(B0, INS, r, c4["M"], O.product(B0), int(c4["Icap"]), 0)
    assert (nD, nI) == (c4["d_records"], c4["i_records"])
    got = sorted((tuple(B0[x] for x in d), tuple(INS[x] for x in i)) for d, i in pairs)
    assert got == _want(c4)
