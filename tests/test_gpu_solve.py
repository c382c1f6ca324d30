"""solve(): the partitioned join against the oracle and the reference's own results."""
import math
import random

import pytest

import oracle as O
from carmichael_frontier_b200 import Solver, Tuning, workloads as W
from carmichael_frontier_b200.solve import Instance

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["fused", "partition"])
def solver(cuda, request):
    return Solver(cuda, tuning=Tuning(strategy=request.param))


def as_lists(pairs):
    return sorted([list(D), list(I)] for D, I in pairs)


def test_config1_two_hits(solver, golden):
    w = W.config1()
    res = solver.solve(w.M, w.Q, w.B0, w.r, w.B)
    g = golden["config1"]
    assert res.residue_pairs == 2 and res.rejected == 0
    assert as_lists(res.pairs) == g["pairs"]
    assert sorted([list(h.D), list(h.I), str(h.n)] for h in res.hits) == g["hits"]
    assert res.n_D == 406 and res.n_I == math.comb(157, 2)


@pytest.mark.parametrize("seed", range(6))
def test_small_instances_vs_exhaustive(solver, seed):
    rng = random.Random(seed)
    M = W.draw_modulus(100 + seed)
    Q = W.eligible_pool(M, 5518)
    k = rng.randint(12, 24)
    r = rng.randint(1, 3)
    Qs = Q[: k + rng.randint(r, 50)]
    B0 = Qs[:k]
    P0 = W.product(B0)
    # a bound that cuts the pair set somewhere in the middle, and an unbounded one
    for B in (P0 * 10 ** rng.randint(0, 12), 1 << 2040):
        res = solver.solve(M, Qs, B0, r, B)
        pairs, hits = O.solve_exhaustive(M, Qs, B0, r, B)
        assert as_lists(res.pairs) == as_lists(pairs)
        assert [(h.D, h.I, h.n) for h in res.hits] == [(tuple(D), tuple(I), n) for D, I, n in hits]
        assert res.rejected == 0


@pytest.mark.parametrize("strategy", ["fused", "partition"])
def test_small_modulus_many_pairs_grows_buffers(cuda, strategy):
    # tiny M: residues collide massively, so partitions and the pair buffer overflow and are regrown
    s = Solver(cuda, tuning=Tuning(d_per_part=64, pair_capacity=16, sigma=0.0, strategy=strategy, dtab_load=11.5))
    M = 2 ** 5 * 3 ** 2 * 5 * 7 * 11 * 13
    Q = W.eligible_pool(M)
    B0 = Q[:20]
    res = s.solve(M, Q, B0, 3, 1 << 2040)
    pairs, hits = O.solve_exhaustive(M, Q, B0, 3, 1 << 2040)
    assert len(pairs) > 200
    assert as_lists(res.pairs) == as_lists(pairs)
    assert len(res.hits) == len(hits) and res.rejected == 0


@pytest.mark.parametrize("idx", [1, 4, 0])
def test_config2_full_size_matches_reference_mitm64(solver, golden, idx):
    g = golden["config2"][idx]
    w = W.Workload(g["name"], g["M"], tuple(g["Q"]), tuple(g["B0"]), g["r"], int(g["B"]))
    res = solver.solve(w.M, w.Q, w.B0, w.r, w.B)
    assert res.n_D == g["d_leaves"] and res.n_I == g["i_leaves"]
    assert res.residue_pairs == g["matches"]
    assert as_lists(res.pairs) == g["pairs"]
    assert sorted([list(h.D), list(h.I), str(h.n)] for h in res.hits) == g["hits"]


def test_positive_control_recovers_previous_incumbent(solver, golden):
    pc = golden["positive_control"]
    N = int(pc["N"])
    res = solver.solve(pc["M"], pc["B0"] + pc["INS"], pc["B0"], pc["r"], N)
    assert res.n_D == math.comb(64, 7) and res.n_I == math.comb(30, 7)
    assert any(h.n == N for h in res.hits)
    assert (tuple(pc["D_need"]), tuple(pc["I_need"])) in set(res.pairs)
    assert res.rejected == 0


def test_edge_cases(solver):
    w = W.config1()
    res = solver.solve(w.M, w.B0, w.B0, 2, w.B)          # no insertions
    assert res.hits == [] and res.n_I == 0
    res = solver.solve(w.M, w.Q, w.B0, 0, w.B)           # radius 0: the base itself
    assert res.n_D == 1
    with pytest.raises(ValueError):
        solver.solve(w.M * 2 ** 40, w.Q, w.B0, 2, w.B)   # M >= 2^62
    with pytest.raises(ValueError):
        solver.solve(w.M, w.Q + (13,), w.B0, 2, w.B)   # 13 divides M


@pytest.mark.parametrize("idx", [1, 4])
def test_config2_with_bloom_first_level(cuda, golden, idx):
    # force the Bloom-filter first level (normally only for D tables larger than L2)
    g = golden["config2"][idx]
    s = Solver(cuda, tuning=Tuning(strategy="fused", l2_table_bytes=0, max_fbits=18))
    res = s.solve(g["M"], g["Q"], g["B0"], g["r"], int(g["B"]))
    assert res.plan["fbits"] > 0
    assert as_lists(res.pairs) == g["pairs"]


def _pair_summary(res):
    return (res.n_D, res.n_I, res.residue_pairs, sorted(res.pairs), [(h.D, h.I, h.n) for h in res.hits])


def test_partitioned_table_build_matches_in_place(cuda, golden):
    # the fused solve's table built by range scatter + shared-memory range builds (default),
    # by the in-place build, and with range capacities too small (rebuilt in place on overflow)
    insts = [Instance.build(g["M"], g["Q"], g["B0"], g["r"], int(g["B"])) for g in golden["config2"][:2]]
    insts.append(Instance.build(*(lambda w: (w.M, w.Q, w.B0, w.r, w.B))(W.config3(2)[1])))
    lim = 1 << 21
    ref = [_pair_summary(Solver(cuda, tuning=Tuning(part_build=False)).solve_instance(x, i_limit=lim))
           for x in insts]
    for tu in (Tuning(part_min_buckets=16), Tuning(part_min_buckets=16, part_lb=9),
               Tuning(part_min_buckets=16, part_sigma=-6.0), Tuning(part_min_buckets=16, dtab_load=12.0)):
        s = Solver(cuda, tuning=tu)
        assert [_pair_summary(s.solve_instance(x, i_limit=lim)) for x in insts] == ref


def test_partitioned_table_build_with_bloom_level(cuda, golden):
    g = golden["config2"][2]
    s = Solver(cuda, tuning=Tuning(strategy="fused", l2_table_bytes=0, max_fbits=18, part_min_buckets=16))
    res = s.solve(g["M"], g["Q"], g["B0"], g["r"], int(g["B"]))
    assert res.plan["fbits"] > 0
    assert as_lists(res.pairs) == g["pairs"]


@pytest.mark.parametrize("M", [5257444553750188800, 12267370625417107200, 17524815179167296000])
def test_moduli_between_2_62_and_2_64(cuda, M):
    # moduli of 63 and 64 bits (the reference's campaign has 4,041 in [2^62, 2^64)): every strategy
    # and the batched portfolio against the exhaustive oracle
    from carmichael_frontier_b200.portfolio import BatchSolver
    assert 1 << 62 <= M < 1 << 64
    Q = W.eligible_pool(M, 5518)
    insts = []
    for k, extra, r in ((20, 25, 2), (18, 22, 3)):
        B0 = Q[:k]
        insts.append(Instance.build(M, Q[:k + extra], B0, r, W.product(B0) * 10 ** 12))
    want = []
    for x in insts:
        pairs, hits = O.solve_exhaustive(x.M, x.B0 + x.INS, x.B0, x.r, x.B)
        want.append((as_lists(pairs), [(tuple(D), tuple(I), n) for D, I, n in hits]))
    for st in ("fused", "partition", "bounded", "auto"):
        s = Solver(cuda, tuning=Tuning(strategy=st))
        for x, (pairs, hits) in zip(insts, want):
            got = s.solve_instance(x)
            assert [(h.D, h.I, h.n) for h in got.hits] == hits, st
            if st in ("fused", "partition"):
                assert as_lists(got.pairs) == pairs, st
    for x, got, (pairs, hits) in zip(insts, BatchSolver(cuda).solve(insts), want):
        assert as_lists(got.pairs) == pairs and [(h.D, h.I, h.n) for h in got.hits] == hits


WIDE_MODULI = [36802111876251321600,           # 2^8 * an odd part of 57 bits: 65 bits
               863845157977978176000,          # 2^9 * an odd part of 61 bits: 70 bits
               5019589575 << 32]               # 2^32 * an odd part of 33 bits: 65 bits


def _packed_residue(M: int, v: int) -> int:
    # the solve path's key of v mod M: (v mod m) << a | v mod 2^a for M = 2^a * m, m odd, mod 2^64
    a = (M & -M).bit_length() - 1
    return (((v % (M >> a)) << a) | (v & ((1 << a) - 1))) & ((1 << 64) - 1)


@pytest.mark.parametrize("M", WIDE_MODULI)
def test_wide_modulus_keys_are_the_residue_keys(cuda, M):
    # moduli of 2^64 and more: every key of both generators (linear, and the tail walker of the
    # fused and partition joins) is the packed exact residue taken mod 2^64, so equal residues meet
    # in the join
    import torch
    from carmichael_frontier_b200 import _lib
    from carmichael_frontier_b200.tables import DeviceTables, unrank_lex
    assert M >= 1 << 64
    lib = _lib.load()
    Q = W.eligible_pool(M, 5518)[:64]
    n = len(Q)
    dt = DeviceTables(cuda)
    rng = random.Random(M & 0xFFFF)
    for r in (2, 3, 5):
        mult = rng.randrange(1, M)
        pool = dt.pool(Q, r, M, mult)
        tail = dt.tail(Q, r, M, mult, pool)
        total = math.comb(n, r)
        count = min(total, 4000)
        lo = rng.randrange(0, total - count + 1)
        keys = torch.empty(count, dtype=torch.uint64, device=cuda)
        ids = torch.empty(count, dtype=torch.uint64, device=cuda)
        _lib.check(lib.cf_gen_subsets(pool.data_ptr(), n, r, lo, count, 1, 0, 0, keys.data_ptr(), ids.data_ptr(),
                                      _lib.stream_handle()), "cf_gen_subsets")
        recs = torch.empty(2 * count, dtype=torch.uint64, device=cuda)
        counts = torch.zeros(1, dtype=torch.int32, device=cuda)
        err = torch.zeros(1, dtype=torch.int32, device=cuda)
        _lib.check(lib.cf_gen_part(pool.data_ptr(), tail.data_ptr(), n, r, lo, count, 0, count, counts.data_ptr(),
                                   recs.data_ptr(), err.data_ptr(), 0, _lib.stream_handle()), "cf_gen_part")
        torch.cuda.synchronize()
        assert int(err.item()) == 0 and int(counts.item()) == count
        want = {}
        for t in range(count):
            S = unrank_lex(lo + t, n, r)
            want[lo + t] = _packed_residue(M, mult * math.prod(Q[i] for i in S))
        lin = dict(zip(ids.cpu().numpy().tolist(), keys.cpu().numpy().tolist()))
        rv = recs.cpu().numpy().reshape(count, 2)
        walk = {int(i): int(k) for k, i in rv}
        assert lin == want and walk == want, r


@pytest.mark.parametrize("M", WIDE_MODULI)
def test_wide_modulus_bounded_records(cuda, M):
    # the bounded producers on moduli of 2^64 and more: the D and I records are the subsets within
    # the product bounds, each keyed by the packed residue (x 2^64 mod m) << a | x mod 2^a, mod 2^64
    import itertools
    from carmichael_frontier_b200.bounded import BoundedGenerator
    from carmichael_frontier_b200.tables import unrank_colex
    a = (M & -M).bit_length() - 1
    m = M >> a

    def packed(v):
        return ((((v % m) << 64) % m) << a | (v & ((1 << a) - 1))) & ((1 << 64) - 1)

    Q = W.eligible_pool(M, 5518)
    B0, INS, r = Q[:24], Q[24:60], 3
    P0 = math.prod(B0)
    gen = BoundedGenerator(cuda)
    dprods = sorted(math.prod(c) for c in itertools.combinations(B0, r))
    Dmin = dprods[len(dprods) // 2]
    k, i, nd = gen.generate_D(B0, r, M, Dmin, bitmask=2)
    got = dict(zip(i.cpu().numpy().tolist(), k.cpu().numpy().tolist()))
    assert nd == len(got) == sum(1 for v in dprods if v >= Dmin)
    for cid, key in got.items():
        v = math.prod(B0[x] for x in unrank_colex(cid, r, len(B0)))
        assert v >= Dmin and key == packed(v)
    iprods = sorted(math.prod(c) for c in itertools.combinations(INS, r))
    Icap = iprods[len(iprods) // 2]
    recs = {}
    for kk, ii in gen.generate_I(INS, r, M, P0, Icap):
        recs.update(zip(ii.cpu().numpy().tolist(), kk.cpu().numpy().tolist()))
    assert len(recs) == sum(1 for v in iprods if v < Icap)
    for cid, key in recs.items():
        v = math.prod(INS[x] for x in unrank_colex(cid, r, len(INS)))
        assert v < Icap and key == packed(P0 * v)


@pytest.mark.parametrize("M", WIDE_MODULI[:2])
def test_wide_modulus_solves(cuda, M):
    # every strategy and the batched portfolio run on moduli of 2^64 and more and agree with the
    # exhaustive oracle (equal residues mod M >= 2^64 do not occur at these sizes; the keys above and
    # the host's exact check of each key match make the join exact)
    from carmichael_frontier_b200 import bsolve
    from carmichael_frontier_b200.portfolio import BatchSolver
    Q = W.eligible_pool(M, 5518)
    insts = []
    for k, extra, r in ((20, 25, 2), (18, 22, 3)):
        B0 = Q[:k]
        insts.append(Instance.build(M, Q[:k + extra], B0, r, W.product(B0) * 10 ** 12))
    assert all(bsolve.applicable(x) for x in insts)
    want = []
    for x in insts:
        pairs, hits = O.solve_exhaustive(x.M, x.B0 + x.INS, x.B0, x.r, x.B)
        want.append((as_lists(pairs), [(tuple(D), tuple(I), n) for D, I, n in hits]))
    for st in ("fused", "partition", "bounded", "auto"):
        s = Solver(cuda, tuning=Tuning(strategy=st))
        for x, (pairs, hits) in zip(insts, want):
            got = s.solve_instance(x)
            assert [(h.D, h.I, h.n) for h in got.hits] == hits, st
            if st in ("fused", "partition"):
                assert as_lists(got.pairs) == pairs, st
                assert got.n_D == math.comb(len(x.B0), x.r) and got.n_I == math.comb(len(x.INS), x.r)
    for x, got, (pairs, hits) in zip(insts, BatchSolver(cuda).solve(insts), want):
        assert as_lists(got.pairs) == pairs and [(h.D, h.I, h.n) for h in got.hits] == hits


def test_modulus_limits(cuda):
    Q = W.eligible_pool(21621600)
    with pytest.raises(ValueError):
        Instance.build(1 << 64, Q, Q[:10], 2, 10 ** 50)          # 2-adic part 2^64: above 2^32
    with pytest.raises(ValueError):
        Instance.build((1 << 63) + 1, [3, 5, 7], [3], 1, 10 ** 50)   # odd part of 2^63 or more


def test_table_uploads_through_the_staging_ring(cuda):
    # asynchronous uploads staged in a small page-locked ring that wraps many times arrive intact,
    # and a table larger than the ring takes the synchronous path
    import numpy as np
    import torch
    from carmichael_frontier_b200.tables import DeviceTables
    dt = DeviceTables(cuda, max_entries=1000, async_upload=True)
    dt.RING_BYTES = 4096
    rng = np.random.default_rng(5)
    want = {}
    for i in range(200):
        a = rng.integers(0, 256, size=int(rng.integers(1, 3000)), dtype=np.uint8)
        want[i] = a
        dt.get(("t", i), lambda a=a: a.copy())
    big = rng.integers(0, 256, size=10000, dtype=np.uint8)
    dt.get(("big",), lambda: big.copy())
    torch.cuda.synchronize()
    for i, a in want.items():
        assert np.array_equal(dt.get(("t", i), None).cpu().numpy(), a)
    assert np.array_equal(dt.get(("big",), None).cpu().numpy(), big)


@pytest.mark.parametrize("strategy,parts", [("fused", 3), ("fused", 100), ("partition", 3)])
def test_i_rank_windows_add_up_to_the_whole_join(cuda, golden, strategy, parts):
    # one modulus split by I-rank window, as shard.run_split splits it over GPUs: the D side complete in
    # every window, the windows' pairs together the reference mitm64's pair set; with 100 windows each
    # (5.9M I ranks) is smaller than the D side (7.6M), so the table is built on the I window (ranks
    # offset by its first rank) and the D side probes it
    from carmichael_frontier_b200 import shard
    g = golden["config2"][1]
    x = Instance.build(g["M"], g["Q"], g["B0"], g["r"], int(g["B"]))
    s = Solver(cuda, tuning=Tuning(strategy=strategy))
    win = shard.windows(g["i_leaves"], parts)
    got = [s.solve_instance(x, i_lo=lo, i_limit=hi) for lo, hi in win]
    assert [r.n_I for r in got] == [hi - lo for lo, hi in win]
    if parts == 100:
        assert all(r.plan["swap"] for r in got)
    m = shard.merge_windows(got)
    assert m.n_D == g["d_leaves"] and m.n_I == g["i_leaves"]
    assert m.residue_pairs == g["matches"] and as_lists(m.pairs) == g["pairs"]
    assert sorted([list(h.D), list(h.I), str(h.n)] for h in m.hits) == g["hits"]
    assert s.solve_instance(x, i_lo=g["i_leaves"], i_limit=g["i_leaves"] + 5).n_I == 0   # an empty window
