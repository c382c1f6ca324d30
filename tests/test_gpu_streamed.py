"""Streamed (out-of-core) join: residue-range partitioning and the partition-by-partition
join through pinned host memory, against numpy and the reference's mitm64 pair sets."""
import math
import random

import numpy as np
import pytest

import oracle as O
from carmichael_frontier_b200 import _lib, workloads as W
from carmichael_frontier_b200.solve import Instance, Solver
from carmichael_frontier_b200.streamed import HostSide, StreamedJoin, streamed_solve

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pbits", [1, 5, 8, 12])
def test_range_partition_matches_numpy(cuda, pbits):
    import torch
    rng = np.random.default_rng(pbits)
    M = W.draw_modulus(40 + pbits)
    n = 300_001
    keys = (rng.integers(0, 2 ** 62, n, dtype=np.uint64) % np.uint64(M)).astype(np.uint64)
    keys[:5] = [0, M - 1, M // 2, 1, M - 2]
    ids = np.arange(n, dtype=np.uint64)
    lib = _lib.load()
    dk = torch.from_numpy(keys.view(np.int64)).to(cuda)
    di = torch.from_numpy(ids.view(np.int64)).to(cuda)
    P = 1 << pbits
    cnt = torch.zeros(P, dtype=torch.int64, device=cuda)
    _lib.check(lib.cf_part_hist(_lib.ptr(dk), n, M, pbits, _lib.ptr(cnt), None), "hist")
    part = np.array([(int(k) << pbits) // M for k in keys], dtype=np.int64)
    want = np.bincount(part, minlength=P)
    assert np.array_equal(cnt.cpu().numpy(), want)
    off = np.concatenate([[0], np.cumsum(want)])
    cur = torch.from_numpy(off[:-1].copy()).to(cuda)
    ok_, oi = torch.empty_like(dk), torch.empty_like(di)
    _lib.check(lib.cf_part_scatter(_lib.ptr(dk), _lib.ptr(di), n, M, pbits, _lib.ptr(cur), _lib.ptr(ok_),
                                   _lib.ptr(oi), None), "scatter")
    assert np.array_equal(cur.cpu().numpy(), off[1:])
    gk = ok_.cpu().numpy().view(np.uint64)
    gi = oi.cpu().numpy().view(np.uint64)
    for p in range(P):
        a, b = off[p], off[p + 1]
        assert np.array_equal(np.sort(gi[a:b]), np.nonzero(part == p)[0].astype(np.uint64))
    assert np.array_equal(keys[gi.astype(np.int64)], gk)


@pytest.mark.parametrize("pbits", [1, 8, 12])
def test_range_partition_of_keys_mod_2_64(cuda, pbits):
    # M = 0 stands for 2^64 (keys of a modulus of 2^64 or more): any u64 key, partition = top bits
    import torch
    rng = np.random.default_rng(100 + pbits)
    n = 200_003
    keys = rng.integers(0, 2 ** 64, n, dtype=np.uint64, endpoint=False)
    keys[:4] = [0, 2 ** 64 - 1, 2 ** 63, 2 ** 63 - 1]
    ids = np.arange(n, dtype=np.uint64)
    lib = _lib.load()
    dk = torch.from_numpy(keys.view(np.int64)).to(cuda)
    di = torch.from_numpy(ids.view(np.int64)).to(cuda)
    P = 1 << pbits
    cnt = torch.zeros(P, dtype=torch.int64, device=cuda)
    _lib.check(lib.cf_part_hist(_lib.ptr(dk), n, 0, pbits, _lib.ptr(cnt), None), "hist")
    part = (keys >> np.uint64(64 - pbits)).astype(np.int64)
    want = np.bincount(part, minlength=P)
    assert np.array_equal(cnt.cpu().numpy(), want)
    off = np.concatenate([[0], np.cumsum(want)])
    cur = torch.from_numpy(off[:-1].copy()).to(cuda)
    ok_, oi = torch.empty_like(dk), torch.empty_like(di)
    _lib.check(lib.cf_part_scatter(_lib.ptr(dk), _lib.ptr(di), n, 0, pbits, _lib.ptr(cur), _lib.ptr(ok_),
                                   _lib.ptr(oi), None), "scatter")
    gi = oi.cpu().numpy().view(np.uint64)
    for p in range(P):
        a, b = off[p], off[p + 1]
        assert np.array_equal(np.sort(gi[a:b]), np.nonzero(part == p)[0].astype(np.uint64))
    assert np.array_equal(keys[gi.astype(np.int64)], ok_.cpu().numpy().view(np.uint64))


def test_streamed_solve_on_a_modulus_above_2_64(cuda):
    # M >= 2^64: the spilled keys are the packed residues mod 2^64, grouped by their top bits, and
    # the streamed solve agrees with the exhaustive oracle
    from carmichael_frontier_b200.tables import unrank_lex
    M = 36802111876251321600
    a = (M & -M).bit_length() - 1
    m = M >> a
    Q = W.eligible_pool(M, 5518)
    for k, extra, r in ((20, 25, 2), (18, 22, 3)):
        inst = Instance.build(M, Q[:k + extra], Q[:k], r, W.product(Q[:k]) * 10 ** 12)
        res, _ = streamed_solve(inst, pbits=4, device=cuda, chunk=1 << 9, piece=1 << 7)
        pairs, hits = O.solve_exhaustive(inst.M, inst.B0 + inst.INS, inst.B0, inst.r, inst.B)
        assert sorted(res.pairs) == sorted(pairs) and [(h.D, h.I, h.n) for h in res.hits] == \
            [(tuple(D), tuple(I), n) for D, I, n in hits]
    side = StreamedJoin(cuda, 4, 1 << 9, 1 << 7).spill(inst.INS, r, M, inst.P0 % M)
    keys, ids = side.keys_np(), side.ids_np()
    assert side.n == len(keys) == len(ids) == math.comb(len(inst.INS), r)
    for p in range(16):
        for j in range(int(side.off[p]), int(side.off[p + 1])):
            v = inst.P0 * math.prod(inst.INS[x] for x in unrank_lex(int(ids[j]), len(inst.INS), r))
            assert int(keys[j]) == ((v % m) << a | (v & ((1 << a) - 1))) & ((1 << 64) - 1)
            assert int(keys[j]) >> 60 == p


@pytest.mark.parametrize("idx", [2, 4])
def test_streamed_solve_matches_reference_mitm64(cuda, golden, idx):
    g = golden["config2"][idx]
    inst = Instance.build(g["M"], g["Q"], g["B0"], g["r"], int(g["B"]))
    # small chunks and pieces: many spill chunks, several pieces per partition
    res, st = streamed_solve(inst, pbits=8, device=cuda, chunk=1 << 22, piece=1 << 18)
    assert res.n_D == g["d_leaves"] and res.n_I == g["i_leaves"]
    assert res.residue_pairs == g["matches"]
    assert sorted([list(D), list(I)] for D, I in res.pairs) == g["pairs"]
    # keys go back to the device (ids stay on the host); partitions with an empty side are skipped
    assert 0 < st["h2d_bytes"] <= 8 * (res.n_D + res.n_I) and st["d2h_bytes"] == 16 * (res.n_D + res.n_I)


def test_streamed_equals_fused_with_many_pairs(cuda):
    # tiny modulus: residues collide everywhere, many pairs per partition
    M = 2 ** 5 * 3 ** 2 * 5 * 7 * 11 * 13
    Q = W.eligible_pool(M)
    inst = Instance.build(M, Q, Q[:20], 3, 1 << 2040)
    res, _ = streamed_solve(inst, pbits=3, device=cuda, chunk=1 << 12, piece=1 << 10)
    pairs, hits = O.solve_exhaustive(M, Q, Q[:20], 3, 1 << 2040)
    assert sorted(res.pairs) == sorted((tuple(D), tuple(I)) for D, I in pairs)
    assert len(res.hits) == len(hits)


def test_host_records_from_the_dumper_format(cuda):
    # sides given as 16-byte {key, id} records on the host (the dumpers' wire format)
    w = W.config1()
    P0 = O.product(w.B0)
    Dk, Did = O.gen_records(w.B0, 2, w.M, 1, 6)
    Ik, Iid = O.gen_records(w.INS, 2, w.M, P0 % w.M, 8)
    D = HostSide.from_records(np.stack([Dk, Did], 1), w.M, 4)
    I = HostSide.from_records(np.stack([Ik, Iid], 1), w.M, 4)
    cand = StreamedJoin(cuda, 4).join(D, I)
    got = sorted((int(D.ids_np()[int(a)]), int(I.ids_np()[int(b)])) for a, b in cand)
    pd, pi = O.join_sorted(*O.sort_side(Dk, Did), *O.sort_side(Ik, Iid))
    assert got == sorted(zip(map(int, pd), map(int, pi))) and len(got) == 2
