"""Product-bounded record producers on the GPU: the filtered I side (igen / idump) and
the Dmin-filtered D side (ddump), exact integer bounds, reference record order.

  generate_I  every r-subset I of the ascending pool with prod(I) < Icap and at most
              hmax primes above `split`: key = P0 * prod(I) mod M, id = colex rank
              (gpu/igen_gpu.py:1-21, src/mitm64_idump_stream2.cpp with IDUMP_RANK=1)
  generate_D  every r-subset D of the ascending base with prod(D) >= Dmin:
              key = prod(D) mod M, id = 6-bit packed indices or a 64-bit mask
              (src/mitm64_ddump.cpp:29-44)

The kernels (csrc/cf_bgen.cu) expand the enumeration tree one level at a time; the
exact bound tables that make every level one contiguous child range per node are
built here with Python integers, like the reference's quotient table
(gpu/igen_gpu.py:92-101).

Keys are canonical residues below M for M < 2^64.  For M >= 2^64 (odd part below 2^63,
2-adic part at most 2^32) a key is the packed residue (x * 2^64 mod m) << a | x mod 2^a
taken mod 2^64: equal residues give equal keys, and callers confirm key matches exactly.
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib
from .tables import DeviceTables, key_of

U128 = 1 << 128


def quotient_table(INS, r: int, Icap: int) -> list[int]:
    """H[t*n + x] = floor((Icap-1) / (a_x ... a_{x+t})) for x + t < n (0 otherwise), 0 <= t < r."""
    n = len(INS)
    top = Icap - 1
    H = [0] * (r * n)
    for t in range(r):
        if t >= n:
            break
        w = math.prod(INS[:t + 1])
        for x in range(n - t):
            if x:
                w = w // INS[x - 1] * INS[x + t]
            H[t * n + x] = top // w
    return H


def dmin_table(B, r: int, Dmin: int) -> list[int]:
    """G[t*n + x] = ceil(Dmin / (b_x b_{x-1} ... b_{x-t})) for x >= t (unused otherwise), 0 <= t < r."""
    n = len(B)
    G = [U128 - 1] * (r * n)
    for t in range(min(r, n)):
        w = math.prod(B[:t + 1])                 # window b_{x-t} ... b_x, slid one prime at a time
        for x in range(t, n):
            if x > t:
                w = w // B[x - t - 1] * B[x]
            G[t * n + x] = -(-Dmin // w) if Dmin > 0 else 0
    return G


def _modulus_ok(M: int) -> bool:
    """M >= 2 with an odd part below 2^63, and a 2-adic part of at most 2^32 when M >= 2^64."""
    a = (M & -M).bit_length() - 1
    return M >= 2 and (M >> a) < 1 << 63 and (M < 1 << 64 or a <= 32)


def _root_key(M: int, mult: int) -> int:
    """Key of the root node: key form of mult mod M, or for M >= 2^64 (whose node keys hold the odd
    part alone) mult * 2^64 mod m, m the odd part of M."""
    if M < 1 << 64:
        return key_of(M, mult % M)
    m = M >> ((M & -M).bit_length() - 1)
    return (mult % m) * (1 << 64) % m


def _cat_u64(parts):
    """Concatenate torch uint64 tensors (through int64 views: torch has no uint64 cat on CUDA)."""
    import torch
    if len(parts) == 1:
        return parts[0]
    return torch.cat([p.view(torch.int64) for p in parts]).view(torch.uint64)


def _u128_pairs(vals) -> np.ndarray:
    """(low, high) u64 words of each value, saturated at 2^128 - 1."""
    m = (1 << 64) - 1
    top = U128 - 1
    vs = [v if v < top else top for v in map(int, vals)]
    a = np.empty(2 * len(vs), dtype=np.uint64)
    a[0::2] = [v & m for v in vs]
    a[1::2] = [v >> 64 for v in vs]
    return a


class BoundedGenerator:
    """Level-by-level bounded enumeration on one device (torch tensors as buffers)."""

    def __init__(self, device=None, max_nodes: int = 1 << 27):
        import torch
        self.torch = torch
        self.lib = _lib.load()
        self.device = torch.device(device if device is not None else "cuda")
        if self.device.type != "cuda":
            raise RuntimeError("bounded generation runs on a CUDA device only")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.tables = DeviceTables(self.device, async_upload=True)   # kernels run on the current stream
        self.max_nodes = max_nodes
        self.launches = 0

    # -- primitives -----------------------------------------------------------
    def _scan(self, cnt, F: int):
        torch = self.torch
        nb = self.lib.cf_scan_tmp_bytes(F)
        ob = (8 * (F + 1) + 255) // 256 * 256            # offsets, then the scan's scratch (one allocation)
        buf = torch.empty(ob + max(nb, 16), dtype=torch.uint8, device=self.device)
        offs = buf[:8 * (F + 1)].view(torch.int64)
        _lib.check(self.lib.cf_scan_u64(_lib.ptr(cnt), F, _lib.ptr(offs), buf.data_ptr() + ob, nb,
                                        _lib.stream_handle()), "cf_scan_u64")
        self.launches += 2
        return offs

    def _frontier(self, side: int, pool, bounds, n: int, r: int, split_idx: int, hmax: int, bitmask: int,
                  xa: int, xb: int, M: int, mult: int, limit: int | None = -1):
        """Nodes at depth r-1 of the block of first indices [xa, xb), their child
        offsets and first child indices; None if a level exceeds the node limit
        (max_nodes by default; None = no limit)."""
        if limit == -1:
            limit = self.max_nodes
        torch, lib, dp = self.torch, self.lib, _lib.ptr
        dev = self.device
        # the root node, read-only: key form of the multiplier, product 1, id 0, meta 0xFFFF
        rt = self.tables.get(("root", M, mult % M), lambda: np.array(
            [_root_key(M, mult), 1, 0, 0, 0xFFFF], dtype=np.uint64).view(np.uint8)).view(torch.int64)
        key, alo, ahi, ids = rt[0:1], rt[1:2], rt[2:3], rt[3:4]
        meta = rt[4:5].view(torch.int32)[:1]
        F = 1
        sh = _lib.stream_handle()
        for d in range(r):
            cx = torch.empty(F + (F + 1) // 2, dtype=torch.int64, device=dev)   # counts, then first indices
            cnt = cx[:F]
            xs = cx[F:].view(torch.int32)[:F]
            _lib.check(lib.cf_bgen_count(side, d, r, n, F, dp(alo), dp(ahi), dp(meta), dp(bounds), split_idx, hmax,
                                         xa, xb, dp(cnt), dp(xs), sh), "cf_bgen_count")
            self.launches += 1
            offs = self._scan(cnt, F)
            total = int(offs[F].item())
            if d == r - 1:
                return dict(F=F, key=key, alo=alo, ahi=ahi, ids=ids, meta=meta, offs=offs, xs=xs, total=total)
            if total == 0:
                return dict(F=0, total=0)
            if limit is not None and total > limit:
                return None
            lv = torch.empty(4 * total + (total + 1) // 2, dtype=torch.int64, device=dev)  # one level's nodes
            nkey, nalo, nahi, nids = (lv[j * total:(j + 1) * total] for j in range(4))
            nmeta = lv[4 * total:].view(torch.int32)[:total]
            _lib.check(lib.cf_bgen_expand(side, d, r, n, F, dp(pool), dp(key), dp(alo), dp(ahi), dp(ids), dp(meta),
                                          dp(offs), dp(xs), split_idx, bitmask, 0, total, dp(nkey), dp(nalo),
                                          dp(nahi), dp(nids), dp(nmeta), sh), "cf_bgen_expand")
            self.launches += 1
            key, alo, ahi, ids, meta, F = nkey, nalo, nahi, nids, nmeta, total
        raise AssertionError("unreachable")

    def _blocks(self, side, pool, bounds, n, r, split_idx, hmax, bitmask, xa, xb, M, mult):
        """Yields the depth-(r-1) frontiers covering first indices [xa, xb), in record
        order; a block whose frontier exceeds max_nodes is halved."""
        fr = self._frontier(side, pool, bounds, n, r, split_idx, hmax, bitmask, xa, xb, M, mult)
        if fr is not None:
            yield fr
            return
        if xb - xa <= 1:
            # a single first index cannot be split further: expand it whole
            yield self._frontier(side, pool, bounds, n, r, split_idx, hmax, bitmask, xa, xb, M, mult, None)
            return
        mid = (xa + xb) // 2
        # I side enumerates first indices ascending, D side descending
        halves = ((xa, mid), (mid, xb)) if side == 0 else ((mid, xb), (xa, mid))
        for a, b in halves:
            yield from self._blocks(side, pool, bounds, n, r, split_idx, hmax, bitmask, a, b, M, mult)

    def _records(self, side, pool, bounds, n, r, split_idx, hmax, bitmask, max_records, M, mult):
        torch, lib, dp = self.torch, self.lib, _lib.ptr
        sh = _lib.stream_handle()
        for fr in self._blocks(side, pool, bounds, n, r, split_idx, hmax, bitmask, 0, n, M, mult):
            total = fr["total"]
            c0 = 0
            while c0 < total:
                cc = min(max_records, total - c0)
                rec = torch.empty(2 * cc, dtype=torch.uint64, device=self.device)
                keys, ids = rec[:cc], rec[cc:]
                _lib.check(lib.cf_bgen_expand(side, r - 1, r, n, fr["F"], dp(pool), dp(fr["key"]), dp(fr["alo"]),
                                              dp(fr["ahi"]), dp(fr["ids"]), dp(fr["meta"]), dp(fr["offs"]),
                                              dp(fr["xs"]), split_idx, bitmask, c0, cc, dp(keys), None, None,
                                              dp(ids), None, sh), "cf_bgen_expand(records)")
                self.launches += 1
                yield keys, ids
                c0 += cc

    # -- the two producers ------------------------------------------------------
    def _setup_I(self, INS, r, M, P0, Icap, split, hmax):
        INS = [int(p) for p in INS]
        n = len(INS)
        assert 1 <= r <= 16 and n <= 1024 and _modulus_ok(M)
        assert all(INS[i] < INS[i + 1] for i in range(n - 1)), "INS must be strictly ascending"
        # the bound table saturates at 2^128 - 1, which is exact while every inner node's product (at
        # most r - 1 primes) stays below 2^128: A <= 2^128 - 1 <= H whenever the true H exceeds it
        assert Icap - 1 < U128 or math.prod(INS[-(r - 1):] if r > 1 else []) < U128, \
            "Icap and the inner products need more than 128 bits"
        if Icap <= 1 or n < r:
            return None
        assert math.comb(n, r) < 1 << 64, "rank ids would overflow u64"
        split_idx = n if split is None else next((i for i, p in enumerate(INS) if p > split), n)
        hmax = r if hmax is None else int(hmax)
        pool = self.tables.pool(INS, r, M, P0 % M)
        bounds = self.tables.get(("igenH", tuple(INS), r, Icap),
                                 lambda: _u128_pairs(quotient_table(INS, r, Icap)).view(np.uint8))
        return INS, n, split_idx, hmax, pool, bounds

    def frontiers_I(self, INS, r: int, M: int, P0: int, Icap: int, split=None, hmax=None):
        """(pool, iterator of depth-(r-1) frontiers) of the filtered I side: the leaves
        are not written, for cf_bgen_probe.  (None, []) when the side is empty."""
        st = self._setup_I(INS, r, M, P0, Icap, split, hmax)
        if st is None:
            return None, iter(())
        INS, n, split_idx, hmax, pool, bounds = st
        return pool, self._blocks(0, pool, bounds, n, r, split_idx, hmax, 0, 0, n, M, P0)

    def generate_I(self, INS, r: int, M: int, P0: int, Icap: int, split=None, hmax=None,
                   max_records: int = 200_000_000):
        """Yields (keys, ids) torch uint64 chunks of the filtered I side; returns the total."""
        st = self._setup_I(INS, r, M, P0, Icap, split, hmax)
        if st is None:
            return 0
        INS, n, split_idx, hmax, pool, bounds = st
        total = 0
        for keys, ids in self._records(0, pool, bounds, n, r, split_idx, hmax, 0, max_records, M, P0):
            total += keys.numel()
            yield keys, ids
        return total

    def generate_D(self, B, r: int, M: int, Dmin: int, bitmask: int = 0, max_records: int = 1 << 62):
        """(keys, ids, count) of the Dmin-filtered D side (torch uint64), ddump's order.
        bitmask: 0 = 6-bit packed ids (a mask when r > 10), 1 = 64-bit index mask (both
        for bases of at most 64 primes, as the dumper), 2 = colex rank (any base)."""
        torch = self.torch
        B = [int(p) for p in B]
        n = len(B)
        mode = int(bitmask)
        if mode == 0 and r > 10:
            mode = 1
        assert mode in (0, 1, 2) and 1 <= r <= 16 and _modulus_ok(M)
        assert n <= (1024 if mode == 2 else 64), "packed and mask ids need a base of at most 64 primes"
        assert all(B[i] < B[i + 1] for i in range(n - 1)), "the base must be strictly ascending"
        if mode == 2:
            assert math.comb(n, r) < 1 << 64, "rank ids would overflow u64"
        empty = (torch.empty(0, dtype=torch.uint64, device=self.device),) * 2 + (0,)
        if n < r or Dmin >= U128:
            return empty
        assert math.prod(B[-r:]) < U128, "products of r base primes must stay below 2^128"
        pool = self.tables.pool(B, r, M, 1)
        bounds = self.tables.get(("ddumpG", tuple(B), r, Dmin),
                                 lambda: _u128_pairs(dmin_table(B, r, max(int(Dmin), 0))).view(np.uint8))
        ks, is_ = [], []
        for k, i in self._records(1, pool, bounds, n, r, n, r, mode, max_records, M, 1):
            ks.append(k)
            is_.append(i)
        if not ks:
            return empty
        k = _cat_u64(ks)
        i = _cat_u64(is_)
        return k, i, int(k.numel())


_gens: dict = {}


def generator(device=None) -> BoundedGenerator:
    import torch
    d = torch.device(device if device is not None else "cuda")
    if d.index is None:
        d = torch.device("cuda", torch.cuda.current_device())
    g = _gens.get(d)
    if g is None:
        g = _gens[d] = BoundedGenerator(d)
    return g
