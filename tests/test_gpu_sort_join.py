"""sort_side / join_sorted drop-ins against the numpy restatements (stable order, every pair)."""
import random

import numpy as np
import pytest
import torch

import oracle as O
from carmichael_frontier_b200 import mitm_gpu2 as G
from carmichael_frontier_b200 import workloads as W

pytestmark = pytest.mark.gpu


def host(t):
    return t.cpu().numpy()


def to_dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint64)).cuda()


@pytest.mark.parametrize("n,bits", [(1, 62), (2, 8), (1000, 62), (8193, 20), (300_000, 62), (2_000_003, 64),
                                    (100_000, 4)])
def test_sort_side_is_numpy_stable_sort(cuda, n, bits):
    rng = np.random.default_rng(n + bits)
    keys = rng.integers(0, 1 << min(bits, 63), size=n, dtype=np.uint64)
    if bits == 64:
        keys |= rng.integers(0, 2, size=n, dtype=np.uint64) << np.uint64(63)
    ids = np.arange(n, dtype=np.uint64) * np.uint64(7919)
    ks, is_ = G.sort_side(to_dev(keys), to_dev(ids))
    ek, ei = O.sort_side(keys, ids)
    assert np.array_equal(host(ks), ek)
    assert np.array_equal(host(is_), ei)    # stability: ties keep input order


@pytest.mark.parametrize("width", [8, 9])
@pytest.mark.parametrize("n,bits", [(2, 9), (4095, 10), (4097, 52), (12_289, 18), (1_000_001, 62), (777_777, 64),
                                    (65_536, 27)])
def test_digit_widths_give_the_numpy_stable_sort(cuda, width, n, bits):
    # every width: odd n (the workspace arrays of odd passes are not 16-byte aligned, so both
    # tile-load variants run), ragged last tiles, a last digit narrower than the width, and
    # passes over constant digits that are skipped
    rng = np.random.default_rng(n * 131 + bits)
    keys = rng.integers(0, 1 << bits, size=n, dtype=np.uint64)
    keys[rng.integers(0, n, size=n // 3)] = keys[0]                  # long runs of one key
    ids = np.arange(n, dtype=np.uint64) ^ np.uint64(0x5DEECE66D)
    ks, is_ = G.sort_side(to_dev(keys), to_dev(ids), digit_bits=width)
    ek, ei = O.sort_side(keys, ids)
    assert np.array_equal(host(ks), ek)
    assert np.array_equal(host(is_), ei)


@pytest.mark.parametrize("width", [8, 9])
@pytest.mark.parametrize("key_bits", [9, 45, 52, 63])
def test_c_entry_with_narrow_key_bits(cuda, width, key_bits):
    # cf_sort_pairs_digits over key_bits bits only (ceil(key_bits / width) passes, no pass above
    # them): keys below 2^key_bits come out in numpy's stable order; the workspace it asks for
    # is the one it needs
    from carmichael_frontier_b200 import _lib
    lib = _lib.load()
    n = 300_007
    rng = np.random.default_rng(key_bits * 10 + width)
    keys = rng.integers(0, 1 << key_bits, size=n, dtype=np.uint64)
    ids = rng.permutation(n).astype(np.uint64)
    kd, idd = to_dev(keys), to_dev(ids)
    nb = lib.cf_sort_digits_tmp_bytes(n, key_bits, width)
    tmp = torch.empty(nb, dtype=torch.uint8, device="cuda")
    _lib.check(lib.cf_sort_pairs_digits(kd.data_ptr(), idd.data_ptr(), n, key_bits, width, tmp.data_ptr(), nb,
                                        _lib.stream_handle()), "sort")
    ek, ei = O.sort_side(keys, ids)
    assert np.array_equal(host(kd), ek) and np.array_equal(host(idd), ei)
    assert lib.cf_sort_pairs_digits(kd.data_ptr(), idd.data_ptr(), n, key_bits, width, tmp.data_ptr(), nb - 1,
                                    _lib.stream_handle()) == _lib.CF_ENOMEM


@pytest.mark.parametrize("width", [8, 9])
def test_more_than_2_30_records(cuda, width):
    # past 2^30 records the look-back's status words are 64-bit (32-bit below): a ragged, odd n with
    # 2^20 distinct keys, so every key repeats about 1000 times and stability is tested everywhere
    free, _ = torch.cuda.mem_get_info()
    if free < (80 << 30):
        pytest.skip("needs about 60 GB of free device memory")
    n = (1 << 30) + 4099
    g = torch.Generator(device="cuda").manual_seed(width)
    keys = torch.randint(0, 1 << 20, (n,), device="cuda", generator=g, dtype=torch.int64)
    ids = torch.arange(n, device="cuda", dtype=torch.int64)
    ks, is_ = G.sort_side(keys.view(torch.uint64), ids.view(torch.uint64), digit_bits=width)
    ks, is_ = ks.view(torch.int64), is_.view(torch.int64)
    assert bool((ks[1:] >= ks[:-1]).all())
    seen = torch.zeros(n, dtype=torch.bool, device="cuda")
    seen[is_] = True
    assert bool(seen.all())                                       # the ids are a permutation
    del seen
    assert torch.equal(ks, keys[is_])                             # each key travelled with its id
    del keys
    eq = ks[1:] == ks[:-1]
    assert bool((is_[1:] > is_[:-1])[eq].all())                  # ties keep input order
    G._ws.clear()                                                 # the 21 GB sort workspace
    del ks, is_, eq
    torch.cuda.empty_cache()


def test_tuned_digit_width_is_used_and_changes_nothing(cuda):
    from carmichael_frontier_b200 import autotune
    sizes = [3000, 70_000, 1 << 20]
    rows = autotune.tune_sort(sizes, key_bits=52, reps=2)
    assert sorted({r["size_class"] for r in rows}) == [n.bit_length() for n in sizes]
    assert all(r["ms"] > 0 and r["digit_bits"] in G.SORT_DIGIT_WIDTHS for r in rows)
    for n in sizes:
        picked = G.sort_digit_bits(n)
        best = min((r for r in rows if r["size_class"] == n.bit_length()), key=lambda r: r["ms"])
        assert picked == best["digit_bits"]
        rng = np.random.default_rng(n)
        keys = rng.integers(0, 1 << 52, size=n, dtype=np.uint64)
        ids = np.arange(n, dtype=np.uint64)
        ks, is_ = G.sort_side(to_dev(keys), to_dev(ids))
        ek, ei = O.sort_side(keys, ids)
        assert np.array_equal(host(ks), ek) and np.array_equal(host(is_), ei)
        G.set_sort_digit_bits(n, None)
        assert G.sort_digit_bits(n) == 8
    with pytest.raises(ValueError):
        G.set_sort_digit_bits(10, 11)
    with pytest.raises(ValueError):
        G.sort_side(to_dev(np.arange(10, dtype=np.uint64)), to_dev(np.arange(10, dtype=np.uint64)), digit_bits=10)


def test_sort_side_all_equal_keys(cuda):
    keys = np.full(50_000, 123456789, dtype=np.uint64)
    ids = np.arange(50_000, dtype=np.uint64)
    for width in G.SORT_DIGIT_WIDTHS:
        ks, is_ = G.sort_side(to_dev(keys), to_dev(ids), digit_bits=width)
        assert np.array_equal(host(is_), ids) and np.array_equal(host(ks), keys)


def test_join_sorted_config1_and_random(cuda):
    w = W.config1()
    P0 = O.product(w.B0)
    Dk, Did = G.generate(list(w.B0), 2, w.M, 1, 6)
    Ik, Iid = G.generate(list(w.INS), 2, w.M, P0 % w.M, 8)
    Dk, Did = G.sort_side(Dk, Did)
    Ik, Iid = G.sort_side(Ik, Iid)
    pd, pi = G.join_sorted(Dk, Did, Ik, Iid)
    ed, ei = O.join_sorted(*O.sort_side(*O.gen_records(w.B0, 2, w.M, 1, 6)),
                           *O.sort_side(*O.gen_records(w.INS, 2, w.M, P0 % w.M, 8)))
    assert np.array_equal(host(pd), ed) and np.array_equal(host(pi), ei)
    assert len(ed) == 2
    # dense duplicates on both sides
    rng = np.random.default_rng(5)
    for nD, nI, span in [(1000, 50_000, 3000), (70_000, 900, 500), (5, 5, 2), (100_000, 100_000, 1 << 40)]:
        dk = np.sort(rng.integers(0, span, nD, dtype=np.uint64))
        ik = np.sort(rng.integers(0, span, nI, dtype=np.uint64))
        did = rng.integers(0, 1 << 62, nD, dtype=np.uint64)
        iid = rng.integers(0, 1 << 62, nI, dtype=np.uint64)
        pd, pi = G.join_sorted(to_dev(dk), to_dev(did), to_dev(ik), to_dev(iid))
        ed, ei = O.join_sorted(dk, did, ik, iid)
        assert np.array_equal(host(pd), ed) and np.array_equal(host(pi), ei)


def test_join_sorted_empty(cuda):
    e = to_dev(np.zeros(0, np.uint64))
    one = to_dev(np.array([5], np.uint64))
    pd, pi = G.join_sorted(e, e, one, one)
    assert pd.numel() == 0 and pi.numel() == 0
    pd, pi = G.join_sorted(one, one, to_dev(np.array([4], np.uint64)), one)
    assert pd.numel() == 0


def test_decode_ids_matches_reference_packing(cuda):
    k, i = G.generate([3, 5, 7, 11, 13], 3, 1000, 1, 6)
    assert G.decode_ids(i, 3, 6)[:2] == [(0, 1, 2), (0, 1, 3)]
