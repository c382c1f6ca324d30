"""Product-bounded producers on the GPU against the oracle restatements of the
reference's dumpers and the reference's own known-answer record counts."""
import hashlib
import math
import random

import numpy as np
import pytest

import oracle as O
from carmichael_frontier_b200 import igen_gpu, workloads as W
from carmichael_frontier_b200.bounded import BoundedGenerator
from carmichael_frontier_b200.tables import unrank_colex

pytestmark = pytest.mark.gpu


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()[:32]


def host(t):
    return t.cpu().numpy() if t.numel() else np.zeros(0, np.uint64)


@pytest.fixture(scope="module")
def gen(cuda):
    return BoundedGenerator(cuda, max_nodes=1 << 22)


def cases(seed, count):
    rng = random.Random(seed)
    for j in range(count):
        M = W.draw_modulus(900 + 17 * seed + j)
        Q = W.eligible_pool(M, 10 ** 5)
        r = rng.randint(1, 7)
        n = rng.randint(max(r, 10), 90)
        while math.comb(n, r) > 2_000_000:          # the oracle enumerates every subset
            n -= 1
        INS = Q[:n]
        lo, hi = math.prod(INS[:r]), math.prod(INS[-r:])
        # a cap anywhere between the smallest and the largest product, and the unbounded one
        Icap = rng.choice([lo, math.isqrt(lo * hi), hi, hi + 1, lo * 50])
        yield M, INS, r, Icap, rng


@pytest.mark.parametrize("seed", range(4))
def test_I_side_equals_idump_records_in_order(gen, seed):
    for M, INS, r, Icap, rng in cases(seed, 8):
        P0 = rng.randrange(1, M)
        split = INS[rng.randrange(len(INS))] if rng.random() < 0.5 else None
        hmax = rng.randint(0, r) if split is not None else None
        split_idx = len(INS) if split is None else next((i for i, p in enumerate(INS) if p > split), len(INS))
        k, i, cnt = O.idump(INS, r, M, P0, Icap, split_idx, r if hmax is None else hmax, rank_ids=True)
        chunks = list(gen.generate_I(INS, r, M, P0, Icap, split, hmax, max_records=777))
        gk = np.concatenate([host(a) for a, _ in chunks]) if chunks else np.zeros(0, np.uint64)
        gi = np.concatenate([host(b) for _, b in chunks]) if chunks else np.zeros(0, np.uint64)
        assert len(gk) == cnt
        assert np.array_equal(gk, k) and np.array_equal(gi, i)


@pytest.mark.parametrize("seed", range(4))
def test_D_side_equals_ddump_records_in_order(gen, seed):
    rng = random.Random(100 + seed)
    for j in range(8):
        M = W.draw_modulus(1300 + 11 * seed + j)
        r = rng.randint(1, 9)
        n = rng.randint(max(r, 8), 64)
        while math.comb(n, r) > 2_000_000:
            n -= 1
        B = W.eligible_pool(M, 5518)[:n]
        r = min(r, len(B))
        lo, hi = math.prod(B[:r]), math.prod(B[-r:])
        Dmin = rng.choice([0, 1, lo, math.isqrt(lo * hi), hi, hi + 1])
        bitmask = rng.random() < 0.3
        k, i, cnt = O.ddump(B, r, M, Dmin, bitmask=bitmask)
        gk, gi, gcnt = gen.generate_D(B, r, M, Dmin, bitmask=bitmask)
        assert gcnt == cnt
        assert np.array_equal(host(gk), k) and np.array_equal(host(gi), i)
        # colex ids (bases beyond 64 primes): same records, same order, ids = colex ranks
        ck, ci, ccnt = gen.generate_D(B, r, M, Dmin, bitmask=2)
        assert ccnt == cnt and np.array_equal(host(ck), k)
        for a, b in zip(host(ci)[:200], i[:200]):
            idx = sorted(x for x in range(64) if (int(b) >> x) & 1) if bitmask or r > 10 else \
                sorted((int(b) >> (6 * q)) & 63 for q in range(r))
            assert unrank_colex(int(a), r, len(B)) == tuple(idx)


@pytest.mark.parametrize("row", [0, 1])
def test_known_answer_counts_at_M0(gen, golden, row):
    # the reference dumpers' record counts and digests at M0 (ksmall base, pool < 82178)
    kat = golden["m0_kat"]
    rr = kat["rows"][row]
    r = rr["r"]
    INS = kat["INS_full"][: rr["n_ins"]]
    P0 = O.product(kat["B0"])
    split = kat["SPLIT"]
    k, i, cnt = igen_gpu.generate(INS, r, kat["M"], P0, int(rr["Icap"]), split, rr["hmax"])
    assert cnt == rr["i_records"]
    kh, ih = host(k), host(i)
    o = np.argsort(ih, kind="stable")
    assert digest(ih[o]) == rr["i_id_digest"] and digest(kh[o]) == rr["i_key_digest"]
    dk, di, dcnt = gen.generate_D(kat["B0"], r, kat["M"], int(rr["Dmin"]))
    assert dcnt == rr["d_records"]
    assert digest(np.sort(host(dk))) == rr["d_key_digest"]
    assert [dcnt, cnt] == kat["documented"][str(r)]


def test_frontier_split_by_first_index(cuda, golden):
    # a tiny node budget forces blocks of first indices; the records and their order stay the same
    kat = golden["m0_kat"]
    rr = kat["rows"][0]
    INS = kat["INS_full"][: rr["n_ins"]]
    P0 = O.product(kat["B0"])
    split = kat["SPLIT"]
    ref = igen_gpu.generate(INS, 4, kat["M"], P0, int(rr["Icap"]), split, rr["hmax"])
    small = BoundedGenerator(cuda, max_nodes=200_000)
    parts = list(small.generate_I(INS, 4, kat["M"], P0, int(rr["Icap"]), split, rr["hmax"], max_records=1 << 20))
    gk = np.concatenate([host(a) for a, _ in parts])
    assert len(parts) > 3 and np.array_equal(gk, host(ref[0]))
