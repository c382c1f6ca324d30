"""The named C entry points of the boundary, called through the C-ABI on the GPU.

cf_join_count / cf_join_emit  against the numpy restatement of join_sorted (gpu/mitm_gpu2.py:107-119),
                              same pairs in the same order, duplicates on both sides;
cf_igen_count / cf_igen_write against the oracle's restatement of mitm64_idump_stream2 (same records,
                              same order) and the reference dumpers' M0 known answer at r = 4,
                              including the workspace-too-small retry;
cf_solve_batch               is the portfolio's only launch path (tests/test_gpu_portfolio.py), and is
                              checked here once more on a small batch against the exhaustive oracle,
                              launched directly and recorded in a CUDA graph.
"""
import ctypes as C
import hashlib
import math
import random

import numpy as np
import pytest
import torch

import oracle as O
from carmichael_frontier_b200 import _lib, tables, workloads as W

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint64).view(np.int64)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("seed", range(3))
def test_join_count_emit_is_join_sorted(cuda, seed):
    lib = _lib.load()
    rng = np.random.default_rng(seed)
    nD, nI = [(1, 1), (5000, 300_001), (200_003, 70_000)][seed]
    Dk = np.sort(rng.integers(0, 4000, nD, dtype=np.uint64))      # dense keys: many equal runs
    Ik = np.sort(rng.integers(0, 4000, nI, dtype=np.uint64))
    Did = rng.integers(0, 1 << 63, nD, dtype=np.uint64)
    Iid = rng.integers(0, 1 << 63, nI, dtype=np.uint64)
    wantD, wantI = O.join_sorted(Dk, Did, Ik, Iid)
    dk, did, ik, iid = _dev(Dk), _dev(Did), _dev(Ik), _dev(Iid)
    tb = lib.cf_join_tmp_bytes(nI)
    tmp = torch.empty(tb, dtype=torch.uint8, device="cuda")
    tot = torch.zeros(1, dtype=torch.int64, device="cuda")
    sh = torch.cuda.current_stream().cuda_stream
    _lib.check(lib.cf_join_count(dk.data_ptr(), nD, ik.data_ptr(), nI, tmp.data_ptr(), tb, tot.data_ptr(), sh),
               "cf_join_count")
    n = int(tot.item())
    assert n == len(wantD)
    oD = torch.empty(max(n, 1), dtype=torch.int64, device="cuda")
    oI = torch.empty_like(oD)
    _lib.check(lib.cf_join_emit(dk.data_ptr(), did.data_ptr(), nD, ik.data_ptr(), iid.data_ptr(), nI, tmp.data_ptr(),
                                oD.data_ptr(), oI.data_ptr(), n, sh), "cf_join_emit")
    assert np.array_equal(_host(oD)[:n], wantD) and np.array_equal(_host(oI)[:n], wantI)


def _igen(lib, INS, r, M, P0, Icap, split_idx, hmax, tmp_bytes=None):
    """Records of the bounded I side through cf_igen_count / cf_igen_write."""
    n = len(INS)
    sh = torch.cuda.current_stream().cuda_stream
    pool = torch.from_numpy(tables.pool_table_host(INS, r, M, P0 % M)).cuda()
    nb = lib.cf_igen_bounds_bytes(n, r)
    hb = np.zeros(nb, dtype=np.uint8)
    ins = np.asarray(INS, dtype=np.uint64)
    _lib.check(lib.cf_igen_bounds(ins.ctypes.data, n, r, Icap & (2 ** 64 - 1), Icap >> 64, hb.ctypes.data, nb),
               "cf_igen_bounds")
    bounds = torch.from_numpy(hb).cuda()
    state = np.zeros(64, dtype=np.uint8)
    total = C.c_uint64(0)
    need = C.c_uint64(0)
    tb = tmp_bytes or lib.cf_igen_tmp_bytes(1 << 16)
    retries = 0
    while True:
        tmp = torch.empty(tb, dtype=torch.uint8, device="cuda")
        rc = lib.cf_igen_count(pool.data_ptr(), bounds.data_ptr(), M, P0 % M, n, r, split_idx, hmax, tmp.data_ptr(),
                               tb, C.byref(total), C.byref(need), state.ctypes.data, sh)
        if rc == _lib.CF_ENOMEM:
            tb = lib.cf_igen_tmp_bytes(need.value)
            retries += 1
            continue
        _lib.check(rc, "cf_igen_count")
        break
    t = total.value
    keys = torch.empty(max(t, 1), dtype=torch.int64, device="cuda")
    ids = torch.empty_like(keys)
    half = t // 2                                   # two write calls: record ranges are independent
    for c0, cc in ((0, half), (half, t - half)):
        _lib.check(lib.cf_igen_write(pool.data_ptr(), n, r, split_idx, tmp.data_ptr(), state.ctypes.data, c0, cc,
                                     keys.data_ptr() + 8 * c0, ids.data_ptr() + 8 * c0, sh), "cf_igen_write")
    return _host(keys)[:t], _host(ids)[:t], retries


@pytest.mark.parametrize("seed", range(3))
def test_igen_count_write_equals_idump(cuda, seed):
    lib = _lib.load()
    rng = random.Random(40 + seed)
    for j in range(6):
        M = W.draw_modulus(700 + 13 * seed + j)
        Q = W.eligible_pool(M, 10 ** 5)
        r = rng.randint(1, 6)
        n = rng.randint(max(r, 8), 70)
        while math.comb(n, r) > 1_500_000:
            n -= 1
        INS = Q[:n]
        lo, hi = math.prod(INS[:r]), math.prod(INS[-r:])
        Icap = rng.choice([lo, math.isqrt(lo * hi), hi + 1])
        P0 = rng.randrange(1, M)
        split_idx = rng.randrange(n + 1)
        hmax = rng.randint(0, r)
        k, i, cnt = O.idump(INS, r, M, P0, Icap, split_idx, hmax, rank_ids=True)
        gk, gi, _ = _igen(lib, INS, r, M, P0, Icap, split_idx, hmax)
        assert len(gk) == cnt and np.array_equal(gk, k) and np.array_equal(gi, i)


def test_igen_count_write_known_answer_at_M0_with_a_small_workspace(cuda, golden):
    lib = _lib.load()
    kat = golden["m0_kat"]
    rr = kat["rows"][0]
    INS = kat["INS_full"][: rr["n_ins"]]
    gk, gi, retries = _igen(lib, INS, rr["r"], kat["M"], O.product(kat["B0"]), int(rr["Icap"]), rr["split_idx"],
                            rr["hmax"], tmp_bytes=lib.cf_igen_tmp_bytes(1024))
    assert retries >= 1 and len(gk) == rr["i_records"]
    dig = lambda a: hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()[:32]  # noqa: E731
    o = np.argsort(gi, kind="stable")
    assert dig(gi[o]) == rr["i_id_digest"] and dig(gk[o]) == rr["i_key_digest"]


def test_solve_batch_small_portfolio_against_the_oracle(cuda):
    from carmichael_frontier_b200.portfolio import BatchSolver
    from carmichael_frontier_b200.solve import Instance
    insts, want = [], []
    for j in range(6):
        M = W.draw_modulus(3100 + j)
        Q = W.eligible_pool(M, 3000)[:40]
        B0 = Q[:14]
        r = 2 + j % 3
        B = math.prod(B0) * 10 ** 6
        insts.append(Instance.build(M, Q, B0, r, B))
        pairs, _hits = O.solve_exhaustive(M, Q, B0, r, B)
        want.append(sorted((tuple(D), tuple(I)) for D, I in pairs))
    for graphs in (False, True):                    # cf_solve_batch launched directly and recorded in a graph
        res = BatchSolver(cuda).solve(insts, graphs=graphs)
        assert [sorted(x.pairs) for x in res] == want
