"""generate() (cf_gen_subsets) against the reference kernel's golden digests and the oracle."""
import hashlib
import math
import random

import numpy as np
import pytest

import oracle as O
from carmichael_frontier_b200 import mitm_gpu2 as G
from carmichael_frontier_b200 import workloads as W

pytestmark = pytest.mark.gpu


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()[:32]


def host(t):
    return t.cpu().numpy()


def test_generate_matches_reference_kernel_digests(cuda, golden):
    for c in golden["gen_records"]:
        k, i = G.generate(c["primes"], c["r"], c["M"], c["mult"], c["bits"], c["lo"], c["hi"])
        assert digest(host(k)) == c["key_digest"], c["name"]
        assert digest(host(i)) == c["id_digest"], c["name"]
        assert [int(x) for x in host(k[:4])] == c["head_keys"]


@pytest.mark.parametrize("r", list(range(1, 11)))
def test_generate_every_radius_vs_oracle(cuda, r):
    rng = random.Random(r)
    w = W.config2(3 + r)
    pool = list(w.B0) if r > 4 else list(w.INS)[:60]
    total = math.comb(len(pool), r)
    for _ in range(3):
        lo = rng.randrange(total)
        hi = min(total, lo + rng.randrange(1, 70_000))
        mult = rng.randrange(w.M)
        k, i = G.generate(pool, r, w.M, mult, 6, lo, hi)
        ok, oi = O.gen_records(pool, r, w.M, mult, 6, lo, hi)
        assert np.array_equal(host(k), ok)
        assert np.array_equal(host(i), oi)


def test_generate_chunks_partition_rank_space(cuda):
    w = W.config1()
    total = math.comb(len(w.INS), 3)
    b = [total * j // 7 for j in range(8)]
    parts = [G.generate(list(w.INS), 3, w.M, 1, 8, lo, hi) for lo, hi in zip(b, b[1:])]
    k_all = np.concatenate([host(k) for k, _ in parts])
    k1, _ = G.generate(list(w.INS), 3, w.M, 1, 8)
    assert np.array_equal(k_all, host(k1))


def test_generate_edge_cases(cuda):
    k, i = G.generate([3, 5, 7], 2, 21621600, 1, 8, 2, 2)
    assert k.numel() == 0 and i.numel() == 0
    k, i = G.generate([3, 5, 7], 3, 21621600, 1, 8)
    assert int(host(k)[0]) == 105 and int(host(i)[0]) == (0 | 1 << 8 | 2 << 16)
    with pytest.raises(AssertionError):
        G.generate([3, 5, 7], 2, 1 << 62, 1, 8)
    with pytest.raises(AssertionError):
        G.generate(list(range(300)), 2, 1000, 1, 8)
    with pytest.raises(AssertionError):
        G.generate([3, 5, 7], 2, 1000, 1, 40)
