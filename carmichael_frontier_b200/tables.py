"""Host-side tables for the kernels: pool tables, screen tables, exact helpers.

Pool tables are filled by the C ABI (``cf_pool_prepare``) into host buffers and
copied to the device once per (prime list, radius, modulus, multiplier); the
copies are cached by content so repeated solves at one modulus reuse them.
"""
from __future__ import annotations

import math
from functools import lru_cache
from math import comb

import numpy as np

from . import _lib

MAX_POOL = 1024
MAX_R = 10
M_LIMIT = 1 << 64          # moduli below this have exact u64 keys; larger ones (odd part < 2^63,
                           # 2-adic part <= 2^32) have keys taken mod 2^64, confirmed exactly


def split_modulus(M: int) -> tuple[int, int]:
    """(odd part m, 2-adic exponent a) of M."""
    a = (M & -M).bit_length() - 1
    return M >> a, a


def wide_modulus(M: int) -> bool:
    """True when keys of M are taken mod 2^64 (M of 2^64 or more), so key matches need an exact check."""
    return M >= M_LIMIT


def pool_table_host(primes, r: int, M: int, mult: int) -> np.ndarray:
    """Pool table (uint8 host array) for the r-subsets of `primes` modulo M."""
    lib = _lib.load()
    n = len(primes)
    nbytes = lib.cf_pool_bytes(n, r)
    if nbytes == 0:
        raise ValueError(f"pool of {n} primes at radius {r} is outside 1..{MAX_POOL} x 1..16")
    pr = np.ascontiguousarray(np.asarray([int(p) for p in primes], dtype=np.uint64))
    out = np.zeros(nbytes, dtype=np.uint8)
    mult = int(mult) % M
    if M < M_LIMIT:
        _lib.check(lib.cf_pool_prepare(pr.ctypes.data, n, r, M, mult, out.ctypes.data, nbytes), "cf_pool_prepare")
    else:
        m, a = split_modulus(M)
        _lib.check(lib.cf_pool_prepare_split(pr.ctypes.data, n, r, m, a, mult % m, mult & ((1 << a) - 1),
                                             out.ctypes.data, nbytes), "cf_pool_prepare_split")
    return out


def _on_stream(stream):
    """Context making `stream` current, or nothing when it already is (the common case)."""
    import contextlib
    import torch
    if stream.cuda_stream == torch._C._cuda_getCurrentRawStream(stream.device_index):
        return contextlib.nullcontext()
    return torch.cuda.stream(stream)


class _PinnedRing:
    """Page-locked staging area for small uploads, allocated once.  A copy takes the next free
    bytes; before the ring wraps, the streams of every copy issued from it since the last wrap
    are synchronised, so no copy reads bytes that are being overwritten."""

    def __init__(self, nbytes: int):
        import torch
        self.buf = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
        self.view = self.buf.numpy()
        self.off = 0
        self.streams: dict = {}

    def upload(self, host, dst, stream) -> bool:
        """Copy host (numpy) into dst (device tensor of the same bytes) on stream without
        waiting; False when host is larger than the ring."""
        import torch
        n = host.nbytes
        if n > len(self.view):
            return False
        if self.off + n > len(self.view):
            for st in self.streams.values():
                st.synchronize()
            self.streams.clear()
            self.off = 0
        a = self.off
        self.view[a:a + n] = host.view(np.uint8).reshape(-1)
        self.off = (a + n + 63) // 64 * 64
        with _on_stream(stream):
            dst.view(torch.uint8).reshape(-1).copy_(self.buf[a:a + n], non_blocking=True)
        self.streams[stream.cuda_stream] = stream
        return True


class DeviceTables:
    """Content-keyed cache of device copies of small host tables.

    stream: the torch stream of the uploads and tail builds (None: the current stream).  With
    async_upload a table is staged in page-locked memory and copied without waiting for the
    device, so kernels queued before it keep running.  An entry remembers the stream it was made
    on and an event after it; a later lookup from another stream (the one the lookup's kernels
    will use: `stream`, or the current stream) makes that stream wait for the event and marks the
    tensor as used there, so entries can be shared by solves on two streams.  Otherwise the copy
    returns when the data is on the device, which any stream may use."""

    RING_BYTES = 4 << 20

    def __init__(self, device, max_entries: int = 64, stream=None, async_upload: bool = False):
        self.device = device
        self.max_entries = max_entries
        self.stream = stream
        self.async_upload = async_upload
        self._ring = None
        self._cache: dict = {}
        self._made: dict = {}          # key -> (raw stream it was made on, event after it)

    def _stream_now(self):
        import torch
        return self.stream if self.stream is not None else torch.cuda.current_stream(self.device)

    def _made_on(self, key, t, s):
        import torch
        ev = torch.cuda.Event()
        ev.record(s)
        self._made[key] = (s.cuda_stream, ev)

    def _use(self, key, t):
        """Order the current stream after the making of entry `key` when it was made on another."""
        made = self._made.get(key)
        if made is None:
            return t
        s = self._stream_now()
        if made[0] != s.cuda_stream:
            s.wait_event(made[1])
            t.record_stream(s)
        return t

    def _insert(self, key, t):
        if len(self._cache) >= self.max_entries:
            old = next(iter(self._cache))
            self._cache.pop(old)
            self._made.pop(old, None)
        self._cache[key] = t

    def get(self, key, make):
        import torch
        t = self._cache.get(key)
        if t is not None:
            return self._use(key, t)
        host = make()
        if self.async_upload:
            s = self._stream_now()
            with _on_stream(s):
                t = torch.empty(host.shape, dtype=torch.from_numpy(host[:0]).dtype, device=self.device)
            if self._ring is None:
                self._ring = _PinnedRing(self.RING_BYTES)
            if not self._ring.upload(host, t, s):
                with _on_stream(s):
                    t.copy_(torch.from_numpy(host), non_blocking=False)
            self._made_on(key, t, s)
        else:
            t = torch.from_numpy(host).to(self.device, non_blocking=False)
        self._insert(key, t)
        return t

    def clear(self):
        """Drop every entry (the next lookups make and upload their tables again)."""
        self._cache.clear()
        self._made.clear()

    def pool(self, primes, r: int, M: int, mult: int):
        key = ("pool", tuple(int(p) for p in primes), r, M, int(mult) % M)
        return self.get(key, lambda: pool_table_host(primes, r, M, mult))

    def tail(self, primes, r: int, M: int, mult: int, pool_dev):
        """Device tail table (b-subset products) of a pool, built on the device once."""
        import torch
        key = ("tail", tuple(int(p) for p in primes), r, M, int(mult) % M)
        t = self._cache.get(key)
        if t is not None:
            return self._use(key, t)
        lib = _lib.load()
        nbytes = lib.cf_tail_bytes(len(primes), r)
        s = self._stream_now()
        with _on_stream(s):
            t = torch.empty(max(nbytes, 16), dtype=torch.uint8, device=self.device)
        _lib.check(lib.cf_build_tail(pool_dev.data_ptr(), len(primes), r, t.data_ptr(),
                                     _lib.stream_handle(self.stream)), "cf_build_tail")
        self._made_on(key, t, s)
        self._insert(key, t)
        return t

    def screen(self, P0: int, B: int, eps: float):
        key = ("screen", P0, B, eps)
        return self.get(key, lambda: screen_table_host(P0, B, eps))


def limbs32(x: int, nlimbs: int | None = None) -> np.ndarray:
    """Little-endian base-2^32 limbs of a non-negative integer."""
    if x < 0:
        raise ValueError("negative")
    n = max(1, (x.bit_length() + 31) // 32) if nlimbs is None else nlimbs
    return np.array([(x >> (32 * i)) & 0xFFFFFFFF for i in range(n)], dtype=np.uint32)


def screen_table_host(P0: int, B: int, eps: float) -> np.ndarray:
    lib = _lib.load()
    if B < 1:
        raise ValueError("size bound B must be >= 1")
    if B.bit_length() > 2048:
        raise ValueError("size bound B must be below 2^2048")
    lb = limbs32(B)
    nbytes = lib.cf_screen_bytes()
    out = np.zeros(nbytes, dtype=np.uint8)
    _lib.check(lib.cf_screen_prepare(lb.ctypes.data, len(lb), math.log2(P0), math.log2(B), eps,
                                     out.ctypes.data, nbytes), "cf_screen_prepare")
    return out


@lru_cache(maxsize=4096)
def ncomb(n: int, r: int) -> int:
    return comb(n, r)


def unrank_lex(rank: int, n: int, r: int) -> tuple[int, ...]:
    """Subset at lexicographic CNS rank (the order of gen_records, gpu/mitm_gpu2.py:40-52)."""
    idx = []
    start = 0
    for pos in range(r):
        rem = r - pos - 1
        for c in range(start, n):
            cnt = ncomb(n - 1 - c, rem)
            if rank < cnt:
                idx.append(c)
                start = c + 1
                break
            rank -= cnt
    return tuple(idx)


def rank_lex(idx, n: int) -> int:
    """Inverse of unrank_lex."""
    r = len(idx)
    rank = 0
    start = 0
    for pos, c in enumerate(idx):
        rem = r - pos - 1
        for c2 in range(start, c):
            rank += ncomb(n - 1 - c2, rem)
        start = c + 1
    return rank


@lru_cache(maxsize=64)
def _colex_columns(r: int, n: int) -> np.ndarray:
    """C(x, t) for x < n, t = 1..r as uint64 columns [r, n] (every colex rank below 2^64)."""
    out = np.zeros((r, n), dtype=np.uint64)
    for t in range(1, r + 1):
        out[t - 1] = np.array([min(comb(x, t), (1 << 64) - 1) for x in range(n)], dtype=np.uint64)
    return out


def unrank_colex_batch(ids, r: int, n: int) -> np.ndarray:
    """unrank_colex of every id in the array ids (ranks below C(n, r) < 2^64): an int64 array
    [len(ids), r] of ascending indices.  Each column is one vectorised search: the largest x with
    C(x, t) <= the remaining rank, t = r .. 1 (C(x, t) increases with x)."""
    v = np.ascontiguousarray(np.asarray(ids, dtype=np.uint64)).copy()
    out = np.zeros((len(v), r), dtype=np.int64)
    cols = _colex_columns(r, n)
    for t in range(r, 0, -1):
        col = cols[t - 1]
        x = np.searchsorted(col, v, side="right").astype(np.int64) - 1
        out[:, t - 1] = x
        v = v - col[x]
    if len(v) and v.any():
        raise ValueError("not a colex rank")
    return out


def unrank_colex(v: int, r: int, n: int) -> tuple[int, ...]:
    """Inverse of the colex rank sum_j C(i_j, j+1) (src/mitm64_idump_stream2.cpp:26-29)."""
    v = int(v)
    idx = []
    x = n - 1
    for j in range(r - 1, -1, -1):
        while ncomb(x, j + 1) > v:
            x -= 1
        idx.append(x)
        v -= ncomb(x, j + 1)
        x -= 1
    if v != 0:
        raise ValueError("not a colex rank")
    return tuple(reversed(idx))


def key_of(M: int, v: int) -> int:
    return int(_lib.load().cf_key_of(M, v % M))


def canon_of(M: int, k: int) -> int:
    return int(_lib.load().cf_canon_of(M, k))
