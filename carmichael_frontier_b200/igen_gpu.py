"""Drop-in for the reference's gpu/igen_gpu.py, on torch CUDA tensors.

Same functions and arguments (gpu/igen_gpu.py:92-162): ``quotient_table``,
``generate_chunks`` (a generator of (keys, ids) chunks whose StopIteration.value
is the total) and ``generate`` (keys, ids, count).  The records are exactly those
of src/mitm64_idump_stream2 with IDUMP_RANK=1 -- every r-subset I of the ascending
INS with prod(I) < Icap and at most hmax primes > split; key = P0*prod(I) mod M,
id = colex rank -- in the same (lexicographic) order.  The kernels are the
level-by-level expansion of csrc/cf_bgen.cu, not a per-thread depth-first walk,
so deep radii balance as well as shallow ones.  Differences: r may be 1..16 (the
reference accepts 3..8) and M must be below 2^64 with an odd part below 2^63 (the reference: 2^64).
"""
from __future__ import annotations

from .bounded import _cat_u64, generator, quotient_table  # noqa: F401  (quotient_table is part of the module's surface)


def generate_chunks(INS, r, M, P0, Icap, split=None, hmax=None, max_records=200_000_000, block_bytes=512 << 20,
                    device=None):
    """Yield (keys, ids) torch uint64 chunks covering exactly the filtered r-subsets of INS;
    the generator's return value is the total record count.  block_bytes is accepted for
    signature compatibility (frontier memory is bounded by the generator's max_nodes)."""
    assert 1 <= r <= 16 and len(INS) <= 1024 and 1 <= M < (1 << 64), "need 1 <= r <= 16, n <= 1024, M < 2^64"
    if Icap <= 1:
        return 0
    gen = generator(device).generate_I(INS, r, M, P0, Icap, split, hmax, max_records=max(1, int(max_records)))
    total = 0
    while True:
        try:
            k, i = next(gen)
        except StopIteration:
            return total
        total += int(k.numel())
        yield k, i


def generate(INS, r, M, P0, Icap, split=None, hmax=None, device=None):
    """Single-shot convenience: concatenated (keys, ids, count)."""
    import torch
    ks, is_ = [], []
    for k, i in generate_chunks(INS, r, M, P0, Icap, split, hmax, max_records=1 << 62, device=device):
        ks.append(k)
        is_.append(i)
    if not ks:
        e = torch.empty(0, dtype=torch.uint64, device=device or "cuda")
        return e, e.clone(), 0
    k = _cat_u64(ks)
    i = _cat_u64(is_)
    return k, i, int(k.numel())
