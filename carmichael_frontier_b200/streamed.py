"""Streamed (out-of-core) join: sides larger than HBM, partitioned by residue range and
streamed through the device from pinned host memory.

At r = 7 over a 160-prime pool the I side has C(96, 7) = 1.19e10 records of 16 bytes
(191 GB), more than a B200 holds.  The materialised plan for such a side:

  spill   generate the side on the device in rank chunks (canonical residue keys,
          lexicographic-rank ids: the reference's 16-byte record), split every
          chunk by residue range p = floor(key * 2^pbits / M) (cf_part_hist +
          cf_part_scatter) and copy each partition's slice into one pinned host
          array per side, at that partition's offset;
  join    for each partition p, copy D_p and I_p (in pieces) to the device on a
          copy stream while partition p-1 is joined on the compute stream: a
          table of D_p (cf_rec_build), probed by I_p (cf_rec_probe); candidate
          positions come back, the keys are compared on the host.

Equal residues fall in the same range, so joining partition by partition finds
every pair.  The reference streams its I side from the C++ dumper through a pipe
and joins every I chunk against every sorted D chunk
(gpu/mitm_gpu_mstar_driver.py:100-118, 241-262); the host arrays here hold the
same 16-byte little-endian records (src/mitm64_idump_stream.cpp:6-12), so a side
can also come from those dumpers (``HostSide.from_records``).  When the sides fit
in HBM the fused join (solve.py) is faster; this path exists for inputs that do
not, or that arrive from the host.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import _lib
from .certify import verify_certificate
from .tables import DeviceTables, ncomb, unrank_lex


def range_partition(keys: np.ndarray, M: int, pbits: int) -> np.ndarray:
    """Residue-range partition floor(key * 2^pbits / M) of uint64 keys below M (M >= 2^64: the top
    pbits bits), exactly, through the partition boundaries ceil(j * M / 2^pbits)."""
    P = 1 << pbits
    Mx = min(int(M), 1 << 64)
    bounds = np.array([-(-(j * Mx) // P) for j in range(1, P)], dtype=np.uint64)
    return np.searchsorted(bounds, np.asarray(keys, dtype=np.uint64), side="right").astype(np.int64)


@dataclass
class HostSide:
    """One side in pinned host memory, grouped by residue-range partition."""
    keys: object            # torch uint64 [N], pinned
    ids: object             # torch uint64 [N], pinned
    off: np.ndarray         # [P + 1] partition offsets
    pbits: int

    @property
    def n(self) -> int:
        return int(self.off[-1])

    def keys_np(self) -> np.ndarray:
        import torch
        return self.keys.view(torch.int64).numpy().view(np.uint64)

    def ids_np(self) -> np.ndarray:
        import torch
        return self.ids.view(torch.int64).numpy().view(np.uint64)

    @staticmethod
    def from_records(rec: np.ndarray, M: int, pbits: int) -> "HostSide":
        """From an (N, 2) uint64 array of {key, id} records (the dumpers' format), on the host."""
        import torch
        keys = rec[:, 0].astype(np.uint64)
        part = range_partition(keys, M, pbits)
        order = np.argsort(part, kind="stable")
        off = np.zeros((1 << pbits) + 1, dtype=np.int64)
        np.add.at(off, part + 1, 1)
        off = np.cumsum(off)
        kt = torch.from_numpy(keys[order].view(np.int64).copy()).pin_memory()
        it = torch.from_numpy(rec[order, 1].astype(np.uint64).view(np.int64).copy()).pin_memory()
        return HostSide(kt.view(torch.uint64), it.view(torch.uint64), off, pbits)


class StreamedJoin:
    def __init__(self, device=None, pbits: int = 8, chunk: int = 1 << 26, piece: int = 1 << 26):
        import torch
        self.torch = torch
        self.lib = _lib.load()
        self.device = torch.device(device if device is not None else "cuda")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.pbits = pbits
        self.chunk = chunk              # records generated per spill step
        self.piece = piece              # records copied per H2D piece in the join
        self.tables = DeviceTables(self.device)
        self.copy_stream = torch.cuda.Stream(self.device)
        self.launches = 0
        self.h2d_bytes = 0
        self.d2h_bytes = 0

    # -- spill ---------------------------------------------------------------------
    def _gen(self, pool, n, r, lo, cnt, keys, ids, sh, canon: int = 1):
        _lib.check(self.lib.cf_gen_subsets(_lib.ptr(pool), n, r, lo, cnt, 1, 0, canon, _lib.ptr(keys), _lib.ptr(ids),
                                           sh), "cf_gen_subsets")
        self.launches += 1

    def host_buffers(self, n: int):
        """Pinned host arrays for n records (keys, ids): allocate once, reuse across spills
        (pinning host memory runs at a few GB/s, far slower than the copies)."""
        import torch
        return (torch.empty(max(n, 1), dtype=torch.int64, pin_memory=True),
                torch.empty(max(n, 1), dtype=torch.int64, pin_memory=True))

    def spill(self, primes, r: int, M: int, mult: int, lo: int = 0, hi: int | None = None,
              out=None) -> HostSide:
        """Generate the records of ranks [lo, hi) on the device and leave them, grouped by
        residue range, in pinned host memory (`out`: arrays from host_buffers, else
        allocated here)."""
        torch = self.torch
        n = len(primes)
        total = ncomb(n, r) if hi is None else hi
        pool = self.tables.pool(primes, r, M, mult)
        # M >= 2^64: packed residue keys taken mod 2^64, partitioned as if M were 2^64
        canon = 0 if M >= 1 << 64 else 1
        sh = _lib.stream_handle()
        cap = min(self.chunk, max(total - lo, 1))
        gk = torch.empty(cap, dtype=torch.uint64, device=self.device)
        gi = torch.empty(cap, dtype=torch.uint64, device=self.device)

        def chunks():
            for c0 in range(lo, total, cap):
                cnt = min(cap, total - c0)
                self._gen(pool, n, r, c0, cnt, gk, gi, sh, canon)
                yield gk[:cnt], gi[:cnt]
        return self.spill_records(chunks, M, out=out, cap=cap)

    def spill_records(self, chunks, M: int, out=None, cap: int | None = None) -> HostSide:
        """Partition a side given as record chunks by residue range into pinned host memory.

        chunks: a callable returning an iterable of (keys, ids) chunks -- uint64 device tensors
        (a producer's output) or host arrays (numpy uint64 or torch tensors: a dumper's
        records), each at most `cap` records; it is called twice, once for the partition sizes
        and once for the scatter, and must yield the same records both times.  Keys below M,
        or any u64 key for M >= 2^64 (partitioned as if M were 2^64)."""
        torch, lib, dp = self.torch, self.lib, _lib.ptr
        P = 1 << self.pbits
        Mp = 0 if M >= 1 << 64 else M
        dev = self.device
        sh = _lib.stream_handle()
        cap = cap or self.chunk
        up = [None, None]

        def on_device(k, i, slot):
            """A chunk as device tensors (host chunks go through one staging buffer pair per slot)."""
            if isinstance(k, torch.Tensor) and k.is_cuda:
                return k.view(torch.uint64), i.view(torch.uint64)
            k = torch.from_numpy(np.ascontiguousarray(k).view(np.int64)) if isinstance(k, np.ndarray) else k
            i = torch.from_numpy(np.ascontiguousarray(i).view(np.int64)) if isinstance(i, np.ndarray) else i
            if up[slot] is None or up[slot][0].numel() < k.numel():
                up[slot] = (torch.empty(max(cap, k.numel()), dtype=torch.int64, device=dev),
                            torch.empty(max(cap, k.numel()), dtype=torch.int64, device=dev))
            uk, ui = up[slot]
            uk[: k.numel()].copy_(k.view(torch.int64))
            ui[: i.numel()].copy_(i.view(torch.int64))
            self.h2d_bytes += 16 * k.numel()
            return uk[: k.numel()].view(torch.uint64), ui[: i.numel()].view(torch.uint64)

        # pass 1: partition sizes of the whole side
        counts = torch.zeros(P, dtype=torch.int64, device=dev)
        N = 0
        for k, i in chunks():
            k, i = on_device(k, i, 0)
            if k.numel():
                _lib.check(lib.cf_part_hist(dp(k), k.numel(), Mp, self.pbits, dp(counts), sh), "cf_part_hist")
                self.launches += 1
            N += k.numel()
        cnts = counts.cpu().numpy()
        off = np.zeros(P + 1, dtype=np.int64)
        off[1:] = np.cumsum(cnts)
        assert off[-1] == N
        if out is not None and out[0].numel() >= N and out[1].numel() >= N:
            hk, hi_ = out
        else:
            hk, hi_ = self.host_buffers(N)
        # pass 2: partition each chunk on the device and copy each partition slice to its host
        # offset on the copy stream; two staging sets, so chunk k+1 is produced and partitioned
        # while chunk k is copied out
        stage = [None, None]
        free = [torch.cuda.Event(), torch.cuda.Event()]
        for e in free:
            e.record()
        cur_host = off[:-1].copy()
        cstream = self.copy_stream
        comp = torch.cuda.current_stream(dev)
        for kk, (k, i) in enumerate(chunks()):
            cnt = k.numel()
            if cnt == 0:
                continue
            comp.wait_event(free[kk & 1])                           # this staging set was copied out
            k, i = on_device(k, i, kk & 1)
            if stage[kk & 1] is None or stage[kk & 1][0].numel() < cnt:
                stage[kk & 1] = (torch.empty(max(cap, cnt), dtype=torch.uint64, device=dev),
                                 torch.empty(max(cap, cnt), dtype=torch.uint64, device=dev))
            sk, si = stage[kk & 1]
            pc = torch.zeros(P, dtype=torch.int64, device=dev)
            _lib.check(lib.cf_part_hist(dp(k), cnt, Mp, self.pbits, dp(pc), sh), "cf_part_hist")
            loc = torch.zeros(P + 1, dtype=torch.int64, device=dev)
            loc[1:] = torch.cumsum(pc, 0)
            cursor = loc[:-1].clone()
            _lib.check(lib.cf_part_scatter(dp(k), dp(i), cnt, Mp, self.pbits, dp(cursor), dp(sk), dp(si), sh),
                       "cf_part_scatter")
            self.launches += 2
            ready = torch.cuda.Event()
            ready.record(comp)
            locs = loc.cpu().numpy()
            with torch.cuda.stream(cstream):
                cstream.wait_event(ready)
                for p in range(P):
                    a, b = int(locs[p]), int(locs[p + 1])
                    if b > a:
                        h = int(cur_host[p])
                        hk[h:h + b - a].copy_(sk[a:b].view(torch.int64), non_blocking=True)
                        hi_[h:h + b - a].copy_(si[a:b].view(torch.int64), non_blocking=True)
                        cur_host[p] += b - a
                free[kk & 1] = torch.cuda.Event()
                free[kk & 1].record(cstream)
            self.d2h_bytes += 16 * cnt
        cstream.synchronize()
        assert np.array_equal(cur_host, off[1:]), "partition sizes changed between the passes"
        return HostSide(hk.view(torch.uint64), hi_.view(torch.uint64), off, self.pbits)

    # -- join ------------------------------------------------------------------------
    def join(self, D: HostSide, I: HostSide, tuning=None) -> np.ndarray:
        """Candidate pairs (global D position, global I position) of equal residues,
        partition by partition; keys compared on the host."""
        from .solve import Tuning, dtab_shape
        torch, lib, dp = self.torch, self.lib, _lib.ptr
        assert D.pbits == I.pbits
        tu = tuning or Tuning()
        dev = self.device
        P = 1 << D.pbits
        sh = _lib.stream_handle()
        comp = torch.cuda.current_stream(dev)
        cstream = self.copy_stream
        maxD = int(np.max(np.diff(D.off))) if D.n else 0
        piece = self.piece
        # two buffer sets: partition p+1 is copied while partition p is joined
        bufs = [dict(dk=torch.empty(max(maxD, 1), dtype=torch.int64, device=dev),
                     ik=torch.empty(max(min(piece, max(I.n, 1)), 1), dtype=torch.int64, device=dev),
                     free=torch.cuda.Event()) for _ in range(2)]
        for b in bufs:
            b["free"].record(comp)
        bbits, fbits = dtab_shape(max(maxD, 1), tu)
        tbytes = lib.cf_dtab_bytes2(bbits, fbits)
        tab = torch.empty(tbytes, dtype=torch.uint8, device=dev)
        misc = torch.zeros(16, dtype=torch.int32, device=dev)
        maxp = 1 << 14
        pairs = torch.empty(maxp * 16, dtype=torch.uint8, device=dev)
        out = []
        steps = []                          # (partition, D range, I piece range)
        for p in range(P):
            d0, d1 = int(D.off[p]), int(D.off[p + 1])
            i0, i1 = int(I.off[p]), int(I.off[p + 1])
            if d1 == d0 or i1 == i0:
                continue
            for a in range(i0, i1, piece):
                steps.append((p, d0, d1, a, min(i1, a + piece), a == i0))
        def issue_copy(k):
            """Copy step k's I piece (and, on a partition's first piece, its D slice) into
            buffer set k % 2 on the copy stream, once that set is free."""
            p, d0, d1, a, b, first = steps[k]
            buf = bufs[k & 1]
            with torch.cuda.stream(cstream):
                cstream.wait_event(buf["free"])
                if first:
                    buf["dk"][: d1 - d0].copy_(D.keys[d0:d1].view(torch.int64), non_blocking=True)
                    self.h2d_bytes += 8 * (d1 - d0)
                buf["ik"][: b - a].copy_(I.keys[a:b].view(torch.int64), non_blocking=True)
                self.h2d_bytes += 8 * (b - a)
                ev = torch.cuda.Event()
                ev.record(cstream)
            return ev

        arrived = issue_copy(0) if steps else None
        for k, (p, d0, d1, a, b, first) in enumerate(steps):
            buf = bufs[k & 1]
            nxt = issue_copy(k + 1) if k + 1 < len(steps) else None     # overlaps this step's join
            comp.wait_event(arrived)
            if first:
                # the table of the partition's D slice serves all of its I pieces
                nb = 1 << bbits
                tab[: 32 * nb].zero_()
                tab[160 * nb: tbytes].zero_()
                misc.zero_()
                _lib.check(lib.cf_rec_build(dp(buf["dk"]), d1 - d0, dp(tab), bbits, fbits, dp(misc) + 4, sh),
                           "cf_rec_build")
                self.launches += 1
            while True:
                misc[0].zero_()
                _lib.check(lib.cf_rec_probe(dp(buf["ik"]), b - a, dp(tab), bbits, fbits, 0, dp(pairs), maxp,
                                            dp(misc), dp(misc) + 4, sh), "cf_rec_probe")
                self.launches += 1
                m = misc[:2].cpu().numpy().view(np.uint32)
                if m[1] & _lib.ERR_PAIR_OVERFLOW:
                    maxp = max(2 * maxp, int(m[0]) + 16)
                    pairs = torch.empty(maxp * 16, dtype=torch.uint8, device=dev)
                    misc[1].zero_()
                    continue
                if m[1]:
                    raise _lib.CfError(_lib.CF_EOVERFLOW, "streamed", f"partition join failed (err {int(m[1]):#x})")
                break
            buf["free"].record(comp)
            np_ = int(m[0])
            if np_:
                pv = pairs[: np_ * 16].cpu().numpy().view(np.uint64).reshape(np_, 2).copy()
                pv[:, 0] += np.uint64(d0)
                pv[:, 1] += np.uint64(a)
                out.append(pv)
            arrived = nxt
        comp.synchronize()
        cand = np.concatenate(out) if out else np.zeros((0, 2), dtype=np.uint64)
        if len(cand):
            dk = D.keys_np()[cand[:, 0].astype(np.int64)]
            ik = I.keys_np()[cand[:, 1].astype(np.int64)]
            cand = cand[dk == ik]
        return cand


def streamed_solve(inst, pbits: int = 8, i_limit: int | None = None, device=None, verify: bool = True,
                   chunk: int = 1 << 26, piece: int = 1 << 26):
    """Solve an instance through the streamed join (both sides spilled to pinned host
    memory, partitioned by residue range, joined partition by partition).  i_limit:
    join only I ranks [0, i_limit).  Returns (SolveResult, stats)."""
    from .solve import Hit, SolveResult
    import time
    sj = StreamedJoin(device, pbits, chunk, piece)
    r, M = inst.r, inst.M
    nD = ncomb(len(inst.B0), r)
    nI = ncomb(len(inst.INS), r)
    if i_limit is not None:
        nI = min(nI, int(i_limit))
    ta = time.perf_counter()
    dbuf, ibuf = sj.host_buffers(nD), sj.host_buffers(nI)
    t0 = time.perf_counter()
    D = sj.spill(inst.B0, r, M, 1, out=dbuf)
    I = sj.spill(inst.INS, r, M, inst.P0 % M, 0, nI, out=ibuf)
    t1 = time.perf_counter()
    cand = sj.join(D, I)
    t2 = time.perf_counter()
    hits, pairs, above = [], [], 0
    dids, iids = D.ids_np(), I.ids_np()
    for dpos, ipos in cand:
        D_ = tuple(inst.B0[x] for x in unrank_lex(int(dids[int(dpos)]), len(inst.B0), r))
        I_ = tuple(inst.INS[x] for x in unrank_lex(int(iids[int(ipos)]), len(inst.INS), r))
        if M >= 1 << 64 and (inst.P0 * math.prod(I_) - math.prod(D_)) % M:
            continue                      # keys equal mod 2^64, residues differ
        pairs.append((D_, I_))
        dset = set(D_)
        fac = tuple(sorted([p for p in inst.B0 if p not in dset] + list(I_)))
        n = math.prod(fac)
        if n > inst.B:
            above += 1
            continue
        ok = (n - 1) % M == 0
        if ok and verify:
            ok, n2, _ = verify_certificate(fac)
            ok = ok and n2 == n
        if ok:
            hits.append(Hit(D_, I_, n, fac))
    hits.sort(key=lambda h: (h.n, h.D, h.I))
    pairs.sort()
    res = SolveResult(hits, nD, nI, len(pairs), len(pairs) - above, above, 0,
                      plan=dict(strategy="streamed", pbits=pbits), pairs=pairs, launches=sj.launches)
    stats = dict(spill_s=t1 - t0, join_s=t2 - t1, pin_alloc_s=t0 - ta, h2d_bytes=sj.h2d_bytes, d2h_bytes=sj.d2h_bytes,
                 host_bytes=16 * (D.n + I.n))
    return res, stats
