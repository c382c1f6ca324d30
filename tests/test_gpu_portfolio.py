"""Batched portfolio: the persistent work-queue kernels against per-modulus solves,
the reference's mitm64 pair sets and the exhaustive oracle."""
import math
import random

import pytest

import oracle as O
from carmichael_frontier_b200 import Solver, workloads as W
from carmichael_frontier_b200.portfolio import BatchSolver, BatchTuning, run_per_modulus, run_plain
from carmichael_frontier_b200.solve import Instance

pytestmark = pytest.mark.gpu


def as_lists(pairs):
    return sorted([list(D), list(I)] for D, I in pairs)


def summary(res):
    return (res.n_D, res.n_I, res.residue_pairs, res.above_bound, res.rejected, as_lists(res.pairs),
            [(h.D, h.I, h.n) for h in res.hits])


def small_portfolio(seed, count):
    """Moduli with small pools, radii 1..4, bounds cutting the pair sets."""
    rng = random.Random(seed)
    out = []
    for j in range(count):
        M = W.draw_modulus(500 + 31 * seed + j)
        Q = W.eligible_pool(M, 5518)
        k = rng.randint(10, 22)
        r = rng.randint(1, 4)
        Qs = Q[: k + rng.randint(r, 40)]
        B0 = Qs[:k]
        B = W.product(B0) * 10 ** rng.randint(0, 14)
        out.append(Instance.build(M, Qs, B0, r, B))
    return out


@pytest.mark.parametrize("seed", range(3))
def test_batched_small_vs_exhaustive(cuda, seed):
    insts = small_portfolio(seed, 24)
    res = BatchSolver(cuda).solve(insts)
    for x, got in zip(insts, res):
        pairs, hits = O.solve_exhaustive(x.M, x.B0 + x.INS, x.B0, x.r, x.B)
        assert as_lists(got.pairs) == as_lists(pairs)
        assert [(h.D, h.I, h.n) for h in got.hits] == [(tuple(D), tuple(I), n) for D, I, n in hits]
        assert got.rejected == 0


def test_batched_config2_matches_reference_mitm64(cuda, golden):
    # five full-size k=64 r=5 moduli in one batch: the reference's own pair sets
    insts = [Instance.build(g["M"], g["Q"], g["B0"], g["r"], int(g["B"])) for g in golden["config2"]]
    res = BatchSolver(cuda).solve(insts)
    for g, got in zip(golden["config2"], res):
        assert got.n_D == g["d_leaves"] and got.n_I == g["i_leaves"]
        assert got.residue_pairs == g["matches"]
        assert as_lists(got.pairs) == g["pairs"]
        assert sorted([list(h.D), list(h.I), str(h.n)] for h in got.hits) == g["hits"]


def test_batched_portfolio_sample_equals_per_modulus_and_plain(cuda):
    # the first moduli of the seeded 1024-modulus portfolio (radii 4..6, pools 120..400),
    # I side limited to a rank prefix; all three forms must agree exactly
    insts = [Instance.build(w.M, w.Q, w.B0, w.r, w.B) for w in W.config3(12)]
    lim = 1 << 20
    got = BatchSolver(cuda).solve(insts, i_limit=lim)
    one = run_per_modulus(insts, i_limit=lim, solver=Solver(cuda))
    plain = run_plain(insts, i_limit=lim, device=cuda)
    for a, b, c in zip(got, one, plain):
        assert summary(a) == summary(b)
        assert (a.residue_pairs, as_lists(a.pairs), [h.n for h in a.hits]) == \
               (c.residue_pairs, as_lists(c.pairs), [h.n for h in c.hits])
        assert a.above_bound == c.above_bound


@pytest.mark.parametrize("overlap", [True, False])
def test_batched_split_budget_graphs_and_overflow(cuda, overlap):
    # many small batches (tiny budget), a pair buffer of 16 that must grow, CUDA-graph replay; with
    # overlap the batches alternate between two arenas and streams, a batch queued before the
    # previous one is collected
    M = 2 ** 5 * 3 ** 2 * 5 * 7 * 11 * 13          # tiny modulus: residues collide massively
    Q = W.eligible_pool(M)
    insts = [Instance.build(M, Q, Q[:20], 3, 1 << 2040)] + small_portfolio(7, 10)
    ref = [summary(x) for x in BatchSolver(cuda, tuning=BatchTuning(overlap=False)).solve(insts)]
    bs = BatchSolver(cuda, tuning=BatchTuning(mem_budget=4096, pair_capacity=16, ticket=64, overlap=overlap))
    prep = bs.prepare(insts)
    assert len(prep.batches) > 3
    for graphs in (False, True, True):
        assert [summary(x) for x in bs.run(prep, graphs=graphs)] == ref
    pairs, _ = O.solve_exhaustive(M, Q, Q[:20], 3, 1 << 2040)
    assert len(pairs) > 200 and as_lists(bs.run(prep)[0].pairs) == as_lists(pairs)


def test_batched_edge_cases(cuda):
    # r = 0, an empty I side, a radius above the batched kernels' maximum (solved one at a time)
    M = 21621600
    Q = W.eligible_pool(M)
    B0 = Q[:29]
    insts = [Instance.build(M, Q, B0, 0, 10 ** 200),
             Instance.build(M, Q[:30], B0, 2, 10 ** 200),          # |INS| = 1 < r: no I records
             Instance.build(M, Q[:40], Q[:12], 9, 1 << 2040),      # r = 9: per-modulus fallback
             Instance.build(M, Q, B0, 2, W.product(B0) * 10 ** 8)]
    bs = BatchSolver(cuda)
    res = bs.solve(insts)
    assert res[1].n_I == 0 and res[1].residue_pairs == 0
    prep = bs.prepare(insts)
    assert prep.fallback == [2]
    one = run_per_modulus(insts, solver=Solver(cuda))
    for a, b in zip(res, one):
        assert summary(a) == summary(b)
    assert len(res[3].hits) == 2


def test_batch_autotuner_keeps_results(cuda):
    from carmichael_frontier_b200.autotune import tune_batch
    insts = small_portfolio(11, 16)
    bs = BatchSolver(cuda)
    prep = bs.prepare(insts)
    ref = [summary(x) for x in bs.run(prep)]
    tu, rows = tune_batch(prep, cuda, reps=1, tickets=(64, 8192), grids=(0, 2))
    assert len(rows) == 4 and all(r["ms"] > 0 for r in rows)
    assert [summary(x) for x in BatchSolver(cuda, tuning=tu).solve(insts)] == ref


def test_batched_partitioned_build_matches_in_place(cuda):
    # tables at 12 records per 16-slot bucket (about one bucket in ten overflows, some of
    # them at the end of a bucket range), tiny whole-table ranges, both range sizes, and the in-place build
    from carmichael_frontier_b200.solve import Tuning
    insts = [Instance.build(w.M, w.Q, w.B0, w.r, w.B) for w in W.config3(6)]
    insts += small_portfolio(3, 8)
    lim = 12 << 17
    dense = Tuning(dtab_load=12.0)
    inplace = BatchSolver(cuda, tuning=BatchTuning(dtab=dense, part_build=False)).solve(insts, i_limit=lim)
    one = run_per_modulus(insts, i_limit=lim, solver=Solver(cuda))
    for lb in (9, 10):
        part = BatchSolver(cuda, tuning=BatchTuning(dtab=dense, part_min_buckets=16, part_lb=lb))
        prep = part.prepare(insts, i_limit=lim)
        assert sum(b.n_part for b in prep.batches) >= 10
        got = part.run(prep)
        assert all(b.use_part for b in prep.batches)
        for a, b, c in zip(got, inplace, one):
            assert summary(a) == summary(b) == summary(c)


def test_batched_partitioned_range_overflow_falls_back(cuda):
    # bucket ranges given less room than they receive: the batch is rebuilt in place
    insts = [Instance.build(w.M, w.Q, w.B0, w.r, w.B) for w in W.config3(3)]
    lim = 1 << 19
    bs = BatchSolver(cuda, tuning=BatchTuning(part_sigma=-6.0, part_min_buckets=16))
    prep = bs.prepare(insts, i_limit=lim)
    got = bs.run(prep, graphs=True)
    assert not any(b.use_part for b in prep.batches if b.n_part)
    ref = BatchSolver(cuda, tuning=BatchTuning(part_build=False)).solve(insts, i_limit=lim)
    for a, b in zip(got, ref):
        assert summary(a) == summary(b)


def test_batched_partitioned_build_with_bloom_level(cuda):
    # the Bloom first level forced on every table (its bits are set by the scatter kernel)
    from carmichael_frontier_b200.solve import Tuning
    insts = [Instance.build(w.M, w.Q, w.B0, w.r, w.B) for w in W.config3(4)]
    lim = 1 << 20
    bloom = Tuning(l2_table_bytes=0, max_fbits=18)
    bs = BatchSolver(cuda, tuning=BatchTuning(dtab=bloom, part_min_buckets=16))
    prep = bs.prepare(insts, i_limit=lim)
    assert all(s is None or s[1] > 0 for s in prep.shapes) and sum(b.n_part for b in prep.batches) == len(insts)
    got = bs.run(prep)
    ref = BatchSolver(cuda, tuning=BatchTuning(part_build=False)).solve(insts, i_limit=lim)
    for a, b in zip(got, ref):
        assert summary(a) == summary(b)


def test_whole_portfolio_moduli_match_reference_mitm64(cuda, golden):
    # whole moduli of the seeded 1024-modulus portfolio (radii 4, 5, 6; pools of 121-272 primes): every
    # D against every I subset, in one batch and one modulus at a time, against the reference's mitm64
    # (its pair set is complete where no two D subsets share a residue: d_res == d_leaves)
    pins = golden["config3_pins"]
    ws = W.config3(1024)
    insts = [Instance.build(ws[g["index"]].M, ws[g["index"]].Q, ws[g["index"]].B0, ws[g["index"]].r, ws[g["index"]].B)
             for g in pins]
    batched = BatchSolver(cuda).solve(insts, graphs=True)
    single = run_per_modulus(insts, solver=Solver(cuda))
    assert {g["r"] for g in pins} == {4, 5, 6}
    for g, a, b in zip(pins, batched, single):
        assert (a.n_D, a.n_I) == (g["d_leaves"], g["i_leaves"])
        assert as_lists(a.pairs) == as_lists(b.pairs)
        if g["d_res"] == g["d_leaves"]:
            assert as_lists(a.pairs) == g["pairs"] and a.residue_pairs == g["matches"]
        else:                                   # mitm64 keeps one D per residue: compare the projection
            assert {tuple(p[1]) for p in as_lists(a.pairs)} == {tuple(p[1]) for p in g["pairs"]}
        assert sorted([list(h.D), list(h.I), str(h.n)] for h in a.hits) == g["hits"]
