"""Python face of the CPU checker (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  It wraps:
  * oracle/cf_oracle.c (libcforacle.so): restatements of gen_records, the full
    pair join, the product-bounded I and D dumpers and mitm64.cpp's join;
  * numpy restatements of sort_side / join_sorted (gpu/mitm_gpu2.py:101-119);
  * an exhaustive small-instance solver in Python integers;
  * the reference's own CPU engines built from source into oracle/_ref/
    (driven through their stdin/stdout formats, src/mitm64.cpp:18-23).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from itertools import combinations
from math import comb

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
_lib = None

u64p = C.POINTER(C.c_uint64)


def lib():
    global _lib
    if _lib is None:
        from build import build_oracle  # type: ignore  (oracle/ is on sys.path for its users)
        path = build_oracle()
        L = C.CDLL(path)
        L.ora_gen_records.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_uint64, C.c_uint64,
                                      C.c_uint64, C.c_void_p, C.c_void_p]
        L.ora_gen_records.restype = None
        L.ora_join_all.argtypes = [C.c_void_p, C.c_int, C.c_uint64, C.c_void_p, C.c_int, C.c_uint64, C.c_int,
                                   C.c_uint64, C.c_void_p, C.c_void_p, C.c_int64]
        L.ora_join_all.restype = C.c_int64
        L.ora_idump.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64,
                                C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_uint64]
        L.ora_idump.restype = C.c_uint64
        L.ora_ddump.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_uint64, C.c_uint64, C.c_uint64, C.c_int,
                                C.c_void_p, C.c_void_p, C.c_uint64]
        L.ora_ddump.restype = C.c_uint64
        L.ora_mitm64.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_uint64, C.c_uint64,
                                 C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p,
                                 C.c_int64, C.c_void_p]
        L.ora_mitm64.restype = C.c_int64
        _lib = L
    return _lib


def _u64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray([int(x) for x in a], dtype=np.uint64))


def _split128(x: int) -> tuple[int, int]:
    if not 0 <= x < 1 << 128:
        raise ValueError("value needs more than 128 bits")
    return x & ((1 << 64) - 1), x >> 64


# ---- restatements --------------------------------------------------------
def gen_records(primes, r, M, mult=1, bits=10, lo=0, hi=None):
    """gen_records (gpu/mitm_gpu2.py:24-98) on the CPU: (keys, ids) numpy uint64."""
    n = len(primes)
    total = comb(n, r)
    hi = total if hi is None else hi
    cnt = hi - lo
    keys = np.zeros(cnt, dtype=np.uint64)
    ids = np.zeros(cnt, dtype=np.uint64)
    if cnt:
        p = _u64(primes)
        lib().ora_gen_records(p.ctypes.data, n, r, bits, M, mult % M, lo, cnt, keys.ctypes.data, ids.ctypes.data)
    return keys, ids


def sort_side(keys, ids):
    """sort_side restated with numpy: stable argsort + gathers."""
    o = np.argsort(keys, kind="stable")
    return keys[o], ids[o]


def join_sorted(Dk, Did, Ik, Iid):
    """join_sorted restated with numpy searchsorted/repeat (gpu/mitm_gpu2.py:107-119)."""
    lo = np.searchsorted(Dk, Ik, side="left")
    hi = np.searchsorted(Dk, Ik, side="right")
    counts = (hi - lo).astype(np.int64)
    total = int(counts.sum())
    if total == 0:
        return np.zeros(0, np.uint64), np.zeros(0, np.uint64)
    cum = np.zeros(len(Ik) + 1, dtype=np.int64)
    np.cumsum(counts, out=cum[1:])
    irow = np.repeat(np.arange(len(Ik), dtype=np.int64), counts)
    within = np.arange(total, dtype=np.int64) - cum[irow]
    dpos = lo[irow] + within
    return Did[dpos], Iid[irow]


def join_all(Dpool, multD, Ipool, multI, r, M, cap=1 << 22):
    """All equal-residue pairs as (D lex rank, I lex rank) arrays (ordered by I rank, D rank)."""
    d = np.zeros(cap, dtype=np.uint64)
    i = np.zeros(cap, dtype=np.uint64)
    Dp, Ip = _u64(Dpool), _u64(Ipool)
    n = lib().ora_join_all(Dp.ctypes.data, len(Dpool), multD % M, Ip.ctypes.data, len(Ipool), multI % M, r, M,
                           d.ctypes.data, i.ctypes.data, cap)
    if n < 0:
        raise MemoryError("ora_join_all")
    if n > cap:
        return join_all(Dpool, multD, Ipool, multI, r, M, cap=int(n))
    return d[:n], i[:n]


def idump(INS, r, M, P0, Icap, split_idx=None, hmax=None, rank_ids=True, cap=None):
    """mitm64_idump_stream2 restated: (keys, ids) in the dumper's depth-first order."""
    n = len(INS)
    split_idx = n if split_idx is None else split_idx
    hmax = 1 << 30 if hmax is None else hmax
    lo, hi = _split128(Icap)
    p = _u64(INS)
    if cap is None:
        cnt = lib().ora_idump(p.ctypes.data, n, r, M, P0 % M, lo, hi, split_idx, hmax, int(rank_ids), None, None, 0)
        cap = int(cnt)
    keys = np.zeros(max(cap, 1), dtype=np.uint64)
    ids = np.zeros(max(cap, 1), dtype=np.uint64)
    cnt = lib().ora_idump(p.ctypes.data, n, r, M, P0 % M, lo, hi, split_idx, hmax, int(rank_ids), keys.ctypes.data,
                          ids.ctypes.data, cap)
    return keys[:min(cnt, cap)], ids[:min(cnt, cap)], int(cnt)


def idump_count(INS, r, M, P0, Icap, split_idx=None, hmax=None):
    n = len(INS)
    lo, hi = _split128(Icap)
    p = _u64(INS)
    return int(lib().ora_idump(p.ctypes.data, n, r, M, P0 % M, lo, hi, n if split_idx is None else split_idx,
                               (1 << 30) if hmax is None else hmax, 1, None, None, 0))


def ddump(B, r, M, Dmin, bitmask=False, cap=None):
    """mitm64_ddump restated: (keys, ids, count) for prod(D) >= Dmin."""
    lo, hi = _split128(Dmin)
    p = _u64(B)
    if cap is None:
        cap = int(lib().ora_ddump(p.ctypes.data, len(B), r, M, lo, hi, int(bitmask), None, None, 0))
    keys = np.zeros(max(cap, 1), dtype=np.uint64)
    ids = np.zeros(max(cap, 1), dtype=np.uint64)
    cnt = lib().ora_ddump(p.ctypes.data, len(B), r, M, lo, hi, int(bitmask), keys.ctypes.data, ids.ctypes.data, cap)
    return keys[:min(cnt, cap)], ids[:min(cnt, cap)], int(cnt)


def mitm64_matches(B0, INS, r, M, P0, Icap, Dmin=1, cap=1 << 20):
    """mitm64.cpp's matches restated: list of (D primes, I primes) and (d_leaves, d_res, i_leaves)."""
    B0 = sorted(B0)
    INS = sorted(INS)
    Bd = B0[::-1]
    b, ins = _u64(B0), _u64(INS)
    d = np.zeros(cap * r, dtype=np.int32)
    i = np.zeros(cap * r, dtype=np.int32)
    st = np.zeros(3, dtype=np.uint64)
    ilo, ihi = _split128(Icap)
    dlo, dhi = _split128(Dmin)
    n = lib().ora_mitm64(b.ctypes.data, len(B0), ins.ctypes.data, len(INS), r, M, P0 % M, ilo, ihi, dlo, dhi,
                         d.ctypes.data, i.ctypes.data, cap, st.ctypes.data)
    out = []
    for k in range(min(n, cap)):
        out.append((tuple(sorted(Bd[x] for x in d[k * r:(k + 1) * r])), tuple(sorted(INS[x] for x in i[k * r:(k + 1) * r]))))
    return out, tuple(int(x) for x in st)


# ---- exhaustive small solver -------------------------------------------
# Order-independent digest of a multiset of 16-byte {key, id} records, for record sets too large to
# hold or sort in one piece (the reference dumpers' outputs at radii 7..13 reach 7.8e8 records):
# three sums mod 2^64 -- of the keys, of the ids and of ((key * C1) xor id) * C2, which ties each key
# to its id.  Chunks are folded with record_digest_add; the tests compute the same sums on the device.
DIGEST_C1 = 0x9E3779B97F4A7C15
DIGEST_C2 = 0xBF58476D1CE4E5B9


def record_digest_add(acc, keys, ids):
    """acc (3 Python ints) plus the records (keys[j], ids[j]) of two uint64 arrays; returns the new acc."""
    k = np.asarray(keys, dtype=np.uint64)
    i = np.asarray(ids, dtype=np.uint64)
    with np.errstate(over="ignore"):
        m = ((k * np.uint64(DIGEST_C1)) ^ i) * np.uint64(DIGEST_C2)
        parts = (int(k.sum(dtype=np.uint64)), int(i.sum(dtype=np.uint64)), int(m.sum(dtype=np.uint64)))
    return tuple((a + b) & 0xFFFFFFFFFFFFFFFF for a, b in zip(acc, parts))


def record_digest_hex(acc) -> str:
    return "".join(f"{x:016x}" for x in acc)


def product(xs) -> int:
    v = 1
    for x in xs:
        v *= x
    return v


def solve_exhaustive(M, Q, B0, r, B):
    """Every (D, I) with prod(S) == 1 mod M (pairs) and the hits with prod(S) <= B; Python integers."""
    B0 = sorted(B0)
    INS = sorted(set(Q) - set(B0))
    P0 = product(B0)
    Pinv = pow(P0, -1, M)
    dres: dict[int, list] = {}
    for D in combinations(B0, r):
        dres.setdefault(product(D) * Pinv % M, []).append(D)
    pairs, hits = [], []
    for I in combinations(INS, r):
        for D in dres.get(product(I) % M, ()):
            pairs.append((D, I))
            n = P0 // product(D) * product(I)
            if n <= B:
                hits.append((D, I, n))
    hits.sort(key=lambda h: (h[2], h[0], h[1]))
    return pairs, hits


def verify_certificate(primes):
    """Independent restatement of ref/ref_carmichael.py:55-72 for the tests."""
    ps = [int(p) for p in primes]
    if len(ps) < 3 or len(set(ps)) != len(ps):
        return False, 0
    bases = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)

    def sprp(n):
        if n < 2:
            return False
        for a in bases:
            if n % a == 0:
                return n == a
        d, s = n - 1, 0
        while d % 2 == 0:
            d //= 2
            s += 1
        for a in bases:
            x = pow(a, d, n)
            if x in (1, n - 1):
                continue
            for _ in range(s - 1):
                x = x * x % n
                if x == n - 1:
                    break
            else:
                return False
        return True

    if not all(sprp(p) for p in ps):
        return False, 0
    n = product(ps)
    return all((n - 1) % (p - 1) == 0 for p in ps), n


# ---- the reference's own CPU engines (built from source into oracle/_ref/) ----
def ref_binary(name: str) -> str | None:
    p = os.path.join(REF_DIR, name)
    return p if os.path.exists(p) else None


def run_ref_mitm64(M, B0, INS, r, P0, Icap, prodDmin=1, threads=None, maxmatch=10 ** 9, timeout=None):
    """Run the reference's mitm64 (stdin format src/mitm64.cpp:18-23); returns (matches, stderr line)."""
    exe = ref_binary("mitm64")
    if exe is None:
        raise FileNotFoundError("oracle/_ref/mitm64 is not built")
    T = threads or os.cpu_count() or 1
    inp = (f"{M} {r} {P0 % M} {Icap} {prodDmin} {T} {maxmatch}\n{len(B0)} {' '.join(map(str, B0))}\n"
           f"{len(INS)} {' '.join(map(str, INS))}\n")
    pr = subprocess.run([exe], input=inp, capture_output=True, text=True, timeout=timeout, check=True)
    out = []
    for line in pr.stdout.splitlines():
        if line.startswith("MATCH"):
            parts = line.split("|")
            D = tuple(sorted(int(x) for x in parts[1].split()[1:]))
            I = tuple(sorted(int(x) for x in parts[2].split()[1:]))
            out.append((D, I))
    return out, pr.stderr.strip()
