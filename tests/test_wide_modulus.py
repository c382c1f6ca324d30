"""Moduli of 2^64 and more (odd part below 2^63, 2-adic part at most 2^32): the split pool
preparation, the instance limits and the host's exact confirmation of key matches (CPU only)."""
import random

import numpy as np
import pytest

from carmichael_frontier_b200 import _lib, bsolve, tables, workloads as W
from carmichael_frontier_b200.solve import RESULT_DTYPE, Instance, finish_rows

WIDE = [36802111876251321600, 863845157977978176000, 5019589575 << 32]


def _split_table(primes, r, m, a, mult):
    lib = _lib.load()
    n = len(primes)
    nbytes = lib.cf_pool_bytes(n, r)
    pr = np.asarray(primes, dtype=np.uint64)
    out = np.zeros(nbytes, dtype=np.uint8)
    rc = lib.cf_pool_prepare_split(pr.ctypes.data, n, r, m, a, mult % m, mult & ((1 << a) - 1),
                                   out.ctypes.data, nbytes)
    return rc, out


@pytest.mark.parametrize("M", [21621600, 9025877244384000, 1768248177696000, 3 * (1 << 32), 135137,
                               ((1 << 63) - 25) * 2])
def test_split_preparation_equals_the_whole_modulus_one(M):
    # below 2^64 the table from (m, a) is byte for byte the table from M
    Q = W.eligible_pool(M, 5518)[:40] or [3, 5, 7, 11]
    Q = [q for q in Q if M % q] or [3, 5, 7, 11]
    a = (M & -M).bit_length() - 1
    rng = random.Random(M)
    for r in (1, 2, 3):
        if r > len(Q):
            continue
        mult = rng.randrange(1, M)
        rc, split = _split_table(Q, r, M >> a, a, mult)
        assert rc == 0
        assert np.array_equal(split, tables.pool_table_host(Q, r, M, mult))


def test_split_preparation_rejects_bad_parts():
    for m, a in ((10, 4), (1 << 63 | 1, 8), (15, 33), (1, 0)):
        rc, _ = _split_table([3, 5, 7], 2, m, a, 1)
        assert rc == _lib.CF_EBADARG
    assert b"odd m below 2^63" in _lib.load().cf_last_error_string()


@pytest.mark.parametrize("M", WIDE)
def test_wide_pool_header(M):
    # the header of a wide modulus: M recorded as 0, the odd part and 2-adic exponent, the fast
    # path's start values from the multiplier's two residues
    a = (M & -M).bit_length() - 1
    m = M >> a
    Q = W.eligible_pool(M, 5518)[:50]
    mult = 987654321987654321987
    w = tables.pool_table_host(Q, 3, M, mult).view("<u8")
    assert int(w[1]) == 0 and int(w[2]) == m and int(w[5]) == a and int(w[6]) == len(Q)
    assert int(w[14]) == 1                                     # every pool prime below 2^31
    assert int(w[15]) == mult % M % m * pow(2, 96, m) % m      # X0 = (mult mod m) 2^(32R) mod m
    assert int(w[16]) == mult % M & ((1 << a) - 1)             # x20 = mult mod 2^a


def test_instance_limits():
    M = WIDE[0]
    Q = W.eligible_pool(M, 5518)
    x = Instance.build(M, Q[:40], Q[:20], 2, 10 ** 90)
    assert x.M == M and tables.wide_modulus(M) and bsolve.applicable(x)
    with pytest.raises(ValueError):
        Instance.build(((1 << 63) + 1) << 4, [3, 5, 7], [3], 1, 10 ** 50)   # odd part of 2^63 or more
    with pytest.raises(ValueError):
        Instance.build(3 << 40, [5, 7, 11], [5], 1, 10 ** 50)              # 2-adic part above 2^32


@pytest.mark.parametrize("strategy", ["fused", "partition"])
def test_key_match_with_different_residues_is_dropped(strategy):
    # a key match of a wide modulus is kept only when P0 * prod(I) == prod(D) (mod M) holds exactly;
    # below 2^64 keys are whole residues and the same row is a pair
    Mw = WIDE[0]
    Q = W.eligible_pool(Mw, 5518)
    xw = Instance.build(Mw, Q[:30], Q[:12], 2, 10 ** 90)
    assert (xw.P0 * xw.INS[0] * xw.INS[1] - xw.B0[0] * xw.B0[1]) % Mw
    row = np.zeros(1, dtype=RESULT_DTYPE)
    row["flags"] = _lib.HIT_KEY_EQUAL
    row["r"] = 2
    row["d_idx"][0, :2] = [0, 1]
    row["i_idx"][0, :2] = [0, 1]
    plan = {"strategy": strategy}
    res = finish_rows(xw, row, 66, 153, plan, verify=True)
    assert res.pairs == [] and res.residue_pairs == 0
    assert res.rejected == (0 if strategy == "fused" else 1)
    Mn = 21621600
    Qn = W.eligible_pool(Mn, 5518)
    xn = Instance.build(Mn, Qn[:30], Qn[:12], 2, 10 ** 90)
    res = finish_rows(xn, row, 66, 153, plan, verify=True)
    assert res.residue_pairs == 1 and res.pairs == [((xn.B0[0], xn.B0[1]), (xn.INS[0], xn.INS[1]))]

