"""Solver.solve_many: solves overlapped with the host's collection of the previous one give the
same results as one solve_instance call per instance, in every path (fused, partition, radius 0,
empty sides, overflow retries) and against the reference's mitm64 pair sets."""
import pytest

import oracle as O
from carmichael_frontier_b200 import Solver, Tuning, workloads as W
from carmichael_frontier_b200.solve import Instance

pytestmark = pytest.mark.gpu


def summary(res):
    return (res.n_D, res.n_I, res.residue_pairs, res.screened, res.above_bound, res.rejected,
            sorted(res.pairs), [(h.D, h.I, h.n) for h in res.hits])


def as_lists(pairs):
    return sorted([list(D), list(I)] for D, I in pairs)


@pytest.mark.parametrize("strategy", ["fused", "partition"])
def test_config2_fixtures_in_one_pipelined_run(cuda, golden, strategy):
    gs = golden["config2"]
    insts = [Instance.build(g["M"], g["Q"], g["B0"], g["r"], int(g["B"])) for g in gs]
    s = Solver(cuda, tuning=Tuning(strategy=strategy))
    marks = []
    out = s.solve_many(insts, marks_list=marks)
    assert len(out) == len(gs) == len(marks)
    for g, res, mk in zip(gs, out, marks):
        assert res.n_D == g["d_leaves"] and res.n_I == g["i_leaves"]
        assert res.residue_pairs == g["matches"]
        assert as_lists(res.pairs) == g["pairs"]
        assert sorted([list(h.D), list(h.I), str(h.n)] for h in res.hits) == g["hits"]
        assert [t for t, _ in mk][0] == "start" and res.launches >= 3


def test_mixed_paths_and_retries_match_one_at_a_time(cuda):
    # tiny pair capacity: most solves overflow their pair buffer and are re-run larger, while the
    # next solve is already queued; radius 0 and an empty I side take the direct paths in between
    w = W.config1()
    M = 2 ** 5 * 3 ** 2 * 5 * 7 * 11 * 13
    Q = W.eligible_pool(M)
    insts = [Instance.build(w.M, w.Q, w.B0, w.r, w.B),
             Instance.build(M, Q, Q[:20], 3, 1 << 2040),
             Instance.build(w.M, w.Q, w.B0, 0, w.B),
             Instance.build(M, Q[:30], Q[:18], 2, 1 << 2040),
             Instance.build(w.M, w.B0, w.B0, 2, w.B),
             Instance.build(M, Q, Q[:22], 2, 1 << 2040)]
    for strategy in ("fused", "partition"):
        tu = Tuning(strategy=strategy, pair_capacity=16, d_per_part=64, sigma=0.0)
        one = [summary(Solver(cuda, tuning=tu).solve_instance(x)) for x in insts]
        many = [summary(r) for r in Solver(cuda, tuning=tu).solve_many(insts, readback_rows=8)]
        assert many == one
    pairs, hits = O.solve_exhaustive(M, Q, Q[:20], 3, 1 << 2040)
    assert as_lists(many[1][6]) == as_lists(pairs) and len(many[1][7]) == len(hits)


def test_i_limit_and_repeated_instances(cuda, golden):
    g = golden["config2"][1]
    x = Instance.build(g["M"], g["Q"], g["B0"], g["r"], int(g["B"]))
    s = Solver(cuda)
    lim = 1 << 22
    ref = summary(s.solve_instance(x, i_limit=lim))
    out = s.solve_many([x, x, x], i_limit=lim)
    assert [summary(r) for r in out] == [ref] * 3


def test_partitioned_builds_pipelined(cuda, golden):
    # the partitioned table build (its descriptor staged in page-locked memory per buffer set) in the
    # pipelined, two-stream sequence, with I windows, against one solve at a time
    gs = golden["config2"][:3]
    insts = [Instance.build(g["M"], g["Q"], g["B0"], g["r"], int(g["B"])) for g in gs]
    insts = insts + insts[::-1]
    lim = 1 << 22
    one = [summary(Solver(cuda, tuning=Tuning(part_build=False)).solve_instance(x, i_limit=lim)) for x in insts]
    s = Solver(cuda, tuning=Tuning(part_min_buckets=16))
    assert [summary(r) for r in s.solve_many(insts, i_limit=lim)] == one
    # a window that starts inside the I side: the pairs with I ranks in [2^21, 2^22) only
    half = [summary(r) for r in s.solve_many(insts, i_limit=lim, i_lo=1 << 21)]
    low = [summary(r) for r in s.solve_many(insts, i_limit=1 << 21)]
    for h, l, o in zip(half, low, one):
        assert h[1] + l[1] == o[1] and sorted(h[6] + l[6]) == o[6]
