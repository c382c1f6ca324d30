"""Drop-in for the reference's gpu/mitm_gpu2.py, on torch CUDA tensors.

Same functions, arguments, outputs and assertions as the reference module
(gpu/mitm_gpu2.py:79-126); arrays are torch ``uint64`` CUDA tensors instead of
CuPy arrays.  Every function runs hand-written sm_100a kernels through the C ABI
(``include/cfmitm.h``):

  generate    -> cf_gen_subsets   (lexicographic rank ranges, canonical residues)
  sort_side   -> cf_sort_pairs_digits (stable LSD onesweep radix sort, keys and ids, tuned digit width)
  join_sorted -> cf_merge_join_runs + host expansion of the (rare) equal runs
"""
from __future__ import annotations

from math import comb

import numpy as np

from . import _lib
from .tables import DeviceTables

_tables: dict = {}
_ws: dict = {}


def _torch():
    import torch
    return torch


def _device(dev=None):
    torch = _torch()
    d = torch.device(dev if dev is not None else "cuda")
    if d.type != "cuda":
        raise RuntimeError("mitm_gpu2 runs on a CUDA device only")
    if d.index is None:
        d = torch.device("cuda", torch.cuda.current_device())
    return d


def _dtables(dev) -> DeviceTables:
    t = _tables.get(dev)
    if t is None:
        t = _tables[dev] = DeviceTables(dev)
    return t


def _workspace(dev, name: str, nbytes: int):
    torch = _torch()
    key = (dev, name)
    t = _ws.get(key)
    if t is None or t.numel() < nbytes:
        t = torch.empty(max(nbytes, 16), dtype=torch.uint8, device=dev)
        _ws[key] = t
    return t


def generate(primes, r: int, M: int, mult: int = 1, bits: int = 10, lo: int = 0, hi=None, device=None):
    """Residue records for the r-combinations of `primes` with CNS rank in [lo, hi).
    Returns torch uint64 (keys, ids); ids pack r indices of `bits` bits each."""
    torch = _torch()
    n = len(primes)
    assert 1 <= r <= 10 and r * bits <= 64, f"r={r}, bits={bits}: need r*bits<=64, r<=10"
    assert n <= (1 << bits), f"pool {n} does not fit {bits}-bit indices"
    assert M < (1 << 62), "M must stay < 2^62 so the residue key fits u64 uniquely"
    total = comb(n, r)
    if hi is None:
        hi = total
    assert 0 <= lo <= hi <= total, (lo, hi, total)
    count = hi - lo
    dev = _device(device)
    keys = torch.empty(count, dtype=torch.uint64, device=dev)
    ids = torch.empty(count, dtype=torch.uint64, device=dev)
    if count == 0:
        return keys, ids
    if M < 2:
        raise ValueError("M must be at least 2")
    pool = _dtables(dev).pool(primes, r, M, mult)
    lib = _lib.load()
    _lib.check(lib.cf_gen_subsets(_lib.ptr(pool), n, r, lo, count, 0, bits, 1, _lib.ptr(keys), _lib.ptr(ids),
                                  _lib.stream_handle()), "generate")
    return keys, ids


SORT_DIGIT_WIDTHS = (8, 9)
_sort_digits: dict[int, int] = {}     # size class (bit length of n) -> digit width picked by the autotuner


def sort_digit_bits(n: int) -> int:
    """Radix digit width sort_side uses for n records: the autotuner's pick for n's size class
    (autotune.tune_sort), else 8."""
    return _sort_digits.get(int(n).bit_length(), 8)


def set_sort_digit_bits(n: int, bits: int | None) -> None:
    """Record the digit width for n's size class (None forgets the class's pick)."""
    if bits is None:
        _sort_digits.pop(int(n).bit_length(), None)
        return
    if bits not in SORT_DIGIT_WIDTHS:
        raise ValueError(f"digit width {bits} not in {SORT_DIGIT_WIDTHS}")
    _sort_digits[int(n).bit_length()] = int(bits)


def sort_side(keys, ids, digit_bits: int | None = None):
    """Sort one side by key (stable LSD radix sort). Returns (sorted_keys, sorted_ids).
    digit_bits (8 or 9) overrides the tuned radix digit width; the result is the same."""
    n = keys.numel()
    ko = keys.contiguous().clone()
    io = ids.contiguous().clone()
    if n <= 1:
        return ko, io
    db = sort_digit_bits(n) if digit_bits is None else int(digit_bits)
    if db not in SORT_DIGIT_WIDTHS:
        raise ValueError(f"digit width {db} not in {SORT_DIGIT_WIDTHS}")
    dev = ko.device
    lib = _lib.load()
    nbytes = lib.cf_sort_digits_tmp_bytes(n, 64, db)
    tmp = _workspace(dev, "sort", nbytes)
    _lib.check(lib.cf_sort_pairs_digits(_lib.ptr(ko), _lib.ptr(io), n, 64, db, _lib.ptr(tmp), nbytes,
                                        _lib.stream_handle()), "sort_side")
    return ko, io


def join_sorted(Dk, Did, Ik, Iid):
    """Sort-merge join of two ALREADY-SORTED sides. Emits EVERY equal-key (D,I) pair."""
    torch = _torch()
    nD, nI = Dk.numel(), Ik.numel()
    dev = Ik.device
    empty = (torch.empty(0, dtype=torch.uint64, device=dev), torch.empty(0, dtype=torch.uint64, device=dev))
    if nD == 0 or nI == 0:
        return empty
    lib = _lib.load()
    run_bytes = lib.cf_merge_run_bytes()
    cap = 1 << 12
    while True:
        runs = _workspace(dev, "runs", cap * run_bytes)
        ctr = _workspace(dev, "runctr", 32)
        ctr.zero_()
        base = _lib.ptr(ctr)
        _lib.check(lib.cf_merge_join_runs(_lib.ptr(Dk), nD, _lib.ptr(Ik), nI, _lib.ptr(runs), cap, base,
                                          base + 8, base + 16, _lib.stream_handle()), "join_sorted")
        c = ctr[:24].cpu().numpy().view(np.uint64)   # synchronises
        nruns, npairs = int(c[0]), int(c[1])
        if nruns <= cap:
            break
        cap = nruns + 16
    if npairs == 0:
        return empty
    rv = runs[: nruns * run_bytes].cpu().numpy().view(np.uint64).reshape(nruns, 3)
    rv = rv[np.argsort(rv[:, 0], kind="stable")]
    irow = np.repeat(rv[:, 0].astype(np.int64), rv[:, 2].astype(np.int64))
    starts = np.repeat(rv[:, 1].astype(np.int64), rv[:, 2].astype(np.int64))
    within = np.arange(len(irow), dtype=np.int64) - np.repeat(np.cumsum(rv[:, 2].astype(np.int64)) - rv[:, 2].astype(np.int64), rv[:, 2].astype(np.int64))
    dpos = torch.from_numpy(starts + within).to(dev)
    ir = torch.from_numpy(irow).to(dev)
    # torch has no uint64 gather on CUDA: gather the same 8-byte words viewed as int64
    return (Did.view(torch.int64)[dpos].view(torch.uint64), Iid.view(torch.int64)[ir].view(torch.uint64))


def decode_ids(ids, r: int, bits: int):
    """Unpack ids -> list of index tuples (host)."""
    if hasattr(ids, "cpu"):
        ids = ids.cpu().numpy()
    mask = (1 << bits) - 1
    return [tuple((int(v) >> (p * bits)) & mask for p in range(r)) for v in ids]
