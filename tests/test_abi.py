"""C-ABI library: loads without a GPU, exports every declared symbol, host helpers are exact."""
import ctypes as C
import math
import os
import random
import re

import numpy as np
import pytest

from carmichael_frontier_b200 import _lib, tables

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    out = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            out += re.findall(r"\b(cf_[a-z0-9_]+)\s*\(", txt)
    return sorted(set(out))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s
    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert set(syms) <= bound


def test_version_and_error_string():
    lib = _lib.load()
    assert lib.cf_version() == 1
    assert isinstance(lib.cf_last_error_string(), bytes)


def test_bad_arguments_fail_loudly_without_gpu():
    lib = _lib.load()
    buf = np.zeros(64, dtype=np.uint8)
    pr = np.array([3, 5, 7], dtype=np.uint64)
    assert lib.cf_pool_prepare(pr.ctypes.data, 3, 2, 1 << 62, 1, buf.ctypes.data, 64) == _lib.CF_EBADARG
    assert b"table buffer too small" in lib.cf_last_error_string() or b"M < 2^62" in lib.cf_last_error_string()
    assert lib.cf_gen_subsets(None, 3, 2, 0, 1, 0, 8, 1, None, None, None) == _lib.CF_EBADARG
    assert lib.cf_join_part(None, None, 1, None, None, 1, 1, 2, 1, 0, None, 0, None, None, None) == _lib.CF_EBADARG
    assert lib.cf_batch_run(0, None, None, 1, 64, None, None, None, 0, None, None, None, 0, None) == _lib.CF_EBADARG
    with pytest.raises(_lib.CfError):
        _lib.check(lib.cf_gen_subsets(None, 3, 2, 0, 1, 0, 8, 1, None, None, None), "probe")


def test_batch_descriptor_layout():
    from carmichael_frontier_b200.portfolio import MOD_DTYPE
    lib = _lib.load()
    assert lib.cf_batch_mod_bytes() == MOD_DTYPE.itemsize == 144
    assert lib.cf_batch_max_r() == 8
    # a ticket that is not a multiple of 32 is rejected before any device call
    one = np.zeros(8, dtype=np.uint64)
    assert lib.cf_batch_run(0, one.ctypes.data, one.ctypes.data, 1, 48, one.ctypes.data, None, None, 0,
                            one.ctypes.data, one.ctypes.data, None, 0, None) == _lib.CF_EBADARG


def test_batch_partitioned_build_constants_and_arguments():
    lib = _lib.load()
    assert (lib.cf_batch_part_buckets(9), lib.cf_batch_part_buckets(10), lib.cf_batch_part_buckets(8)) == (512, 1024, 0)
    assert lib.cf_batch_part_tile() == 4064
    assert lib.cf_batch_part_max_ranges() == 2048
    assert lib.cf_batch_ovf_bytes() == 24
    one = np.zeros(8, dtype=np.uint64)
    p = one.ctypes.data
    # bad phase, missing queue or tickets, missing overflow counter: rejected before any device call
    assert lib.cf_batch_part(3, p, p, 1, p, p, 1, p, p, 10, 0, 0, None) == _lib.CF_EBADARG
    assert lib.cf_batch_part(0, p, None, 1, p, None, 0, None, p, 10, 0, 0, None) == _lib.CF_EBADARG
    assert lib.cf_batch_part(1, p, p, 1, None, p, 1, p, p, 10, 0, 0, None) == _lib.CF_EBADARG
    assert lib.cf_batch_part(1, p, p, 1, p, p, 1, p, p, 11, 0, 0, None) == _lib.CF_EBADARG   # range size
    assert lib.cf_batch_part(2, p, None, 1, None, p, 1, None, p, 10, 0, 0, None) == _lib.CF_EBADARG
    assert lib.cf_batch_part(0, p, p, 0, p, None, 0, None, p, 10, 0, 0, None) == _lib.CF_EBADARG
    assert lib.cf_batch_part(0, p, p, 1, p, None, 0, None, p, 10, 9, 0, None) == _lib.CF_EBADARG   # radius


def _hostkey(M, v):
    a = (M & -M).bit_length() - 1
    m = M >> a
    X = (v % m) * pow(2, 64, m) % m if m > 1 else 0
    return (X << a) | (v & ((1 << a) - 1))


@pytest.mark.parametrize("M", [21621600, 9025877244384000, 1768248177696000, (1 << 62) - 2, 3 * (1 << 50),
                               1 << 40, 135137, 2, 6])
def test_key_form_is_a_bijection_and_round_trips(M):
    rng = random.Random(M)
    for _ in range(200):
        v = rng.randrange(M)
        k = tables.key_of(M, v)
        assert k == _hostkey(M, v)
        assert 0 <= k < M
        assert tables.canon_of(M, k) == v


@pytest.mark.parametrize("M", [21621600, 9025877244384000, (1 << 62) - 2, 3 * (1 << 50), 1 << 40, 135137, 6])
def test_key_product_is_the_residue_product(M):
    # cf_key_mul runs the kernels' Montgomery/CRT product (same inline code) on the host
    lib = _lib.load()
    rng = random.Random(M + 1)
    for _ in range(300):
        x, y = rng.randrange(M), rng.randrange(M)
        k = lib.cf_key_mul(M, tables.key_of(M, x), tables.key_of(M, y))
        assert tables.canon_of(M, k) == x * y % M


def test_pool_table_layout():
    lib = _lib.load()
    primes = [11, 13, 17, 19, 23, 29, 31]
    M = 21621600
    t = tables.pool_table_host(primes, 3, M, 5)
    w = t.view(np.uint64)
    assert w[0] == 0x43464d49544d3031
    assert int(w[1]) == M and int(w[5]) == 5 and int(w[6]) == 7 and int(w[7]) == 3   # M, a, n, R
    assert int(w[8]) == tables.key_of(M, 5)                 # mult_key
    assert int(w[9]) == math.comb(7, 3)                     # total
    n = 7
    pkey = w[32:32 + n]
    assert [int(x) for x in pkey] == [tables.key_of(M, p) for p in primes]
    assert [int(x) for x in w[32 + n:32 + 2 * n]] == primes
    lg = w[32 + 2 * n:32 + 3 * n].view(np.float64)
    assert np.allclose(lg, np.log2(primes), rtol=0, atol=1e-15)
    binom = w[32 + 3 * n:].reshape(n + 1, 4)
    for x in range(n + 1):
        for y in range(4):
            assert int(binom[x, y]) == math.comb(x, y)


@pytest.mark.parametrize("M", [21621600, 9025877244384000, 1768248177696000, (1 << 62) - 2, 3 * (1 << 50),
                               1 << 40, 135137, 6, 2])
def test_fast_path_product_is_the_crt_residue(M):
    # the solve path's lazy 32-bit Montgomery product, run on the host, against Python integers
    lib = _lib.load()
    a = (M & -M).bit_length() - 1
    m = M >> a
    rng = random.Random(M + 7)
    for _ in range(300):
        x, y = rng.randrange(1, 1 << 31), rng.randrange(1, 1 << 31)
        v = x * y % M
        assert lib.cf_key32_mul(M, x, y) == ((v % m) << a) | (v & ((1 << a) - 1))


def test_screen_table():
    lib = _lib.load()
    B = 10 ** 148
    t = tables.screen_table_host(3 ** 300, B, 1e-6)
    assert len(t) == lib.cf_screen_bytes()
    d = t[:24].view(np.float64)
    assert abs(d[0] - 300 * math.log2(3)) < 1e-9 and abs(d[1] - 148 * math.log2(10)) < 1e-9 and d[2] == 1e-6
    with pytest.raises(ValueError):
        tables.screen_table_host(3, 1 << 3000, 1e-6)


def test_unrank_rank_lex_round_trip():
    for n, r in [(10, 3), (29, 2), (64, 5), (150, 5)]:
        total = math.comb(n, r)
        for rank in [0, 1, total // 3, total - 1]:
            idx = tables.unrank_lex(rank, n, r)
            assert list(idx) == sorted(set(idx)) and len(idx) == r
            assert tables.rank_lex(idx, n) == rank
    assert tables.unrank_lex(0, 10, 3) == (0, 1, 2)
    assert tables.unrank_lex(math.comb(10, 3) - 1, 10, 3) == (7, 8, 9)


def test_igen_bound_table_equals_the_python_definition():
    from carmichael_frontier_b200.bounded import _u128_pairs, quotient_table
    lib = _lib.load()
    rng = random.Random(5)
    for _ in range(20):
        n = rng.randint(3, 60)
        r = rng.randint(1, min(n, 9))
        INS = sorted(rng.sample(range(3, 50_000, 2), n))
        Icap = rng.choice([1, 2, math.prod(INS[:r]), math.prod(INS[-r:]) + 1, (1 << 128) - 5, rng.randrange(1 << 100)])
        nb = lib.cf_igen_bounds_bytes(n, r)
        out = np.zeros(nb, dtype=np.uint8)
        ins = np.asarray(INS, dtype=np.uint64)
        _lib.check(lib.cf_igen_bounds(ins.ctypes.data, n, r, Icap & (2 ** 64 - 1), Icap >> 64, out.ctypes.data, nb),
                   "cf_igen_bounds")
        want = _u128_pairs(quotient_table(INS, r, Icap))
        assert np.array_equal(out.view(np.uint64), want), (n, r, Icap)
    bad = np.asarray([5, 3], dtype=np.uint64)
    assert lib.cf_igen_bounds(bad.ctypes.data, 2, 1, 100, 0, out.ctypes.data, 64) == _lib.CF_EBADARG


def test_named_entry_points_reject_bad_arguments_without_gpu():
    lib = _lib.load()
    assert lib.cf_join_count(None, 1, None, 1, None, 0, None, None) == _lib.CF_EBADARG
    assert lib.cf_join_emit(None, None, 1, None, None, 1, None, None, None, 1, None) == _lib.CF_EBADARG
    assert lib.cf_igen_count(None, None, 10, 1, 5, 2, 5, 2, None, 0, None, None, None, None) == _lib.CF_EBADARG
    st = np.zeros(64, dtype=np.uint8)
    assert lib.cf_igen_write(st.ctypes.data, 5, 2, 5, st.ctypes.data, st.ctypes.data, 0, 1, None, None, None) \
        == _lib.CF_EBADARG                      # a state that cf_igen_count did not write
    assert lib.cf_solve_batch(None, None) == _lib.CF_EBADARG
    q = _lib.CfBatchQueue()
    assert lib.cf_solve_batch(C.byref(q), None) == _lib.CF_EBADARG
    assert lib.cf_igen_tmp_bytes(1 << 20) > lib.cf_igen_tmp_bytes(1 << 10) > 0
    assert lib.cf_join_tmp_bytes(1000) >= 16 * 1000
    assert lib.cf_dtab_build3(None, None, 5, 2, 0, 10, None, 10, 0, 1, None, None) == _lib.CF_EBADARG
    buf = np.zeros(64, dtype=np.uint8)
    assert lib.cf_rec_build_keyform(buf.ctypes.data, 4, buf.ctypes.data, 10, 0, None, buf.ctypes.data, None) \
        == _lib.CF_EBADARG                      # no pool to take the modulus from
    assert lib.cf_bgen_probe_keyform(2, 10, 0, None, None, None, None, None, 0, 1, None, 10, 0, None, 0, None, None,
                                     None) == _lib.CF_EBADARG


def test_sort_digit_widths_workspace_and_arguments():
    # the workspace of the digit-width sort: ceil(key_bits / width) passes of 2^width bins each;
    # the 8-bit workspace over 64 bits is cf_sort_pairs' own
    lib = _lib.load()
    n = 1 << 20
    tiles = n // 4096
    for bits, width in ((64, 8), (64, 9), (52, 9), (52, 8), (1, 9)):
        npass = -(-bits // width)
        want = 16 * n + 16 * (npass << width) + 8 * tiles * (npass << width) + 8 * 4 + 64
        assert lib.cf_sort_digits_tmp_bytes(n, bits, width) == want
    assert lib.cf_sort_digits_tmp_bytes(n, 64, 8) == lib.cf_sort_tmp_bytes(n)
    assert lib.cf_sort_digits_tmp_bytes(n, 64, 10) == 0 and lib.cf_sort_digits_tmp_bytes(n, 0, 8) == 0
    buf = np.zeros(64, dtype=np.uint8)
    p = buf.ctypes.data
    assert lib.cf_sort_pairs_digits(p, p, 100, 64, 7, p, 64, None) == _lib.CF_EBADARG
    assert b"digit_bits" in lib.cf_last_error_string()
    assert lib.cf_sort_pairs_digits(None, p, 100, 64, 9, p, 64, None) == _lib.CF_EBADARG
    assert lib.cf_sort_pairs_digits(p, p, 100, 65, 9, p, 64, None) == _lib.CF_EBADARG
    assert lib.cf_sort_pairs_digits(p, p, 100, 64, 9, p, 64, None) == _lib.CF_ENOMEM   # before any device work
    assert lib.cf_sort_pairs_digits(p, p, 1, 64, 9, p, 64, None) == _lib.CF_OK          # nothing to sort


def test_ddump_bound_table_equals_the_python_definition():
    from carmichael_frontier_b200.bounded import _u128_pairs, dmin_table
    lib = _lib.load()
    rng = random.Random(6)
    for _ in range(20):
        n = rng.randint(3, 64)
        r = rng.randint(1, min(n, 10))
        B = sorted(rng.sample(range(3, 5_000, 2), n))
        Dmin = rng.choice([0, 1, math.prod(B[:r]), math.prod(B[-r:]), math.prod(B[-r:]) + 1,
                           rng.randrange(1, 1 << 100)])
        nb = lib.cf_ddump_bounds_bytes(n, r)
        out = np.zeros(nb, dtype=np.uint8)
        b = np.asarray(B, dtype=np.uint64)
        _lib.check(lib.cf_ddump_bounds(b.ctypes.data, n, r, Dmin & (2 ** 64 - 1), Dmin >> 64, out.ctypes.data, nb),
                   "cf_ddump_bounds")
        want = _u128_pairs(dmin_table(B, r, Dmin)).reshape(r, n, 2)
        got = out.view(np.uint64).reshape(r, n, 2)
        for t in range(r):                              # entries x < t are never read
            assert np.array_equal(got[t, t:], want[t, t:]), (n, r, Dmin, t)


def test_sort_digit_width_classes_without_gpu():
    # the tuner groups side sizes by bit length (sort_side's lookup key) and times the largest of each
    from carmichael_frontier_b200 import autotune, mitm_gpu2 as G
    assert autotune.sort_size_classes([0, 1, 3000, 4000, 70_000, 65_536, 1 << 20, (1 << 21) - 1]) == \
        {12: 4000, 17: 70_000, 21: (1 << 21) - 1}
    assert autotune.sort_size_classes([]) == {}
    n = 123_457
    assert G.sort_digit_bits(n) == 8                      # untuned classes use 8-bit digits
    G.set_sort_digit_bits(n, 9)
    assert G.sort_digit_bits(n + 1000) == 9 and G.sort_digit_bits(2 * n) == 8
    G.set_sort_digit_bits(n, None)
    assert G.sort_digit_bits(n) == 8
    with pytest.raises(ValueError):
        G.set_sort_digit_bits(n, 10)
    with pytest.raises(ValueError):
        autotune.tune_sort([n], widths=(8, 10))
