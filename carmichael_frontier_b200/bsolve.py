"""Product-bounded solve: prune both sides by the size bound before the join.

A hit S = (B0 \\ D) u I needs prod(S) = P0 * prod(I) / prod(D) <= B.  With
Dmax = the product of the r largest base primes and Imin = the product of the r
smallest insertion primes this gives the reference driver's two filters
(gpu/mitm_gpu_mstar_driver.py:189-203, with U = B + 1):

    prod(I) <  Icap = min(prod of the r largest INS + 1, floor(B * Dmax / P0) + 1)
    prod(D) >= Dmin = ceil(P0 * Imin / B)

The filtered sides come from the bounded producers (csrc/cf_bgen.cu: the igen /
idump and ddump records) and are joined through the record table of
csrc/cf_rec_join.cu -- built on the D records with the I leaves probing it as
they are generated (csrc/cf_bgen_probe.cu), or built on the I records when those
are fewer -- and every equal-key pair is checked exactly on the host (prod(S) <= B, prod(S) == 1 mod M, certificate), as run_instance does
(:241-262).  The hit set equals the unpruned join's: pruning removes only
subsets that no hit can contain.  Where the bound prunes hard (B = prod(B0) *
10^4, the serving workload) the sides are a tiny fraction of C(n, r).
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib
from .bounded import U128
from .certify import verify_certificate
from .tables import pool_table_host, unrank_colex, unrank_colex_batch, wide_modulus

RANK_LIMIT = 1 << 32          # positions in the join table are 32-bit


def caps(inst) -> tuple[int, int]:
    """(Icap, Dmin) of an instance: exclusive I-product cap, inclusive D-product floor."""
    r, P0, B = inst.r, inst.P0, inst.B
    Dmax = math.prod(inst.B0[-r:])
    topI = math.prod(inst.INS[-r:])
    Icap = min(topI + 1, B * Dmax // P0 + 1)
    Imin = math.prod(inst.INS[:r])
    Dmin = -(-(P0 * Imin) // B)
    return Icap, Dmin


def applicable(inst) -> bool:
    """The bounded producers need 128-bit products (and r >= 1, both sides non-empty)."""
    if inst.r < 1 or len(inst.B0) < inst.r or len(inst.INS) < inst.r:
        return False
    Icap, Dmin = caps(inst)
    return Icap - 1 < U128 and math.prod(inst.B0[-inst.r:]) < U128 and math.comb(len(inst.INS), inst.r) < 1 << 64 \
        and math.comb(len(inst.B0), inst.r) < 1 << 64


def bounds_fit(B0, INS, r: int, Icap: int) -> bool:
    """True when the bounded producers can run an instance given by its sides and exclusive I cap:
    1 <= r <= 16, both sides hold r primes, at most 1024 primes each, the products of r base primes
    below 2^128, the I cap below 2^128 or else the products of r - 1 insertion primes below 2^128
    (the I bound table then saturates exactly), and colex ids of either side below 2^64.  The
    reference's GPU producer stops at an I cap of 2^128 (gpu/igen_gpu.py:83,103-105) and its driver
    sends such instances to a host join (gpu/mitm_gpu_mstar_driver.py:150-183,207)."""
    B0, INS = sorted(B0), list(INS)
    if not (1 <= r <= 16) or len(B0) < r or len(INS) < r or len(B0) > 1024 or len(INS) > 1024:
        return False
    inner_fits = Icap - 1 < U128 or math.prod(INS[-(r - 1):] if r > 1 else []) < U128
    return inner_fits and math.prod(B0[-r:]) < U128 and math.comb(len(INS), r) < 1 << 64 \
        and math.comb(len(B0), r) < 1 << 64


def prunes(inst) -> bool:
    """True when the bound removes part of either side (else the fused join is cheaper)."""
    r = inst.r
    Icap, Dmin = caps(inst)
    return Icap <= math.prod(inst.INS[-r:]) or Dmin > math.prod(inst.B0[:r])


class BoundedSolve:
    """Solves one instance with the bounded producers and a record-table join.

    The D side (Dmin filter) is materialised.  The I side (Icap filter) is expanded
    to its last level; when its leaves outnumber the D records they are never
    written: cf_bgen_probe computes each leaf and probes a table of the D records.
    Otherwise the I leaves are written and the table is built on them."""

    LEAF_CHUNK = 1 << 30          # I leaves per probe launch
    WIDE_LEAF_CHUNK = 1 << 26     # I leaves written per chunk for M >= 2^64 (16 bytes each)

    def __init__(self, solver):
        from .bounded import BoundedGenerator
        self.s = solver
        self.torch = solver.torch
        self.lib = solver.lib
        self.gen = BoundedGenerator(solver.device, max_nodes=solver.tuning.max_nodes)
        self.native = True                  # one C call per instance (cf_bounded_join) where it applies
        self._native_bytes = 256 << 20
        self._native_out = 1 << 12
        self._stage = None                  # page-locked staging of one instance's tables

    def _table(self, keys, n: int, plan: dict, keyform_pool=None):
        """Record table of keys[0..n): canonical residues, or, with keyform_pool (a device pool table),
        their key forms under that pool's modulus (probed by cf_bgen_probe_keyform)."""
        from .solve import dtab_shape
        torch, lib, dp = self.torch, self.lib, _lib.ptr
        if n >= RANK_LIMIT:
            raise _lib.CfError(_lib.CF_EOVERFLOW, "bounded", "table side has 2^32 records or more")
        bbits, fbits = dtab_shape(n, self.s.tuning)
        plan.update(bbits=bbits, fbits=fbits)
        tbytes = lib.cf_dtab_bytes2(bbits, fbits)
        tab = self.s._buf("btab", tbytes)
        nbk = 1 << bbits
        tab[: 32 * nbk].zero_()
        tab[160 * nbk: tbytes].zero_()
        self.misc.zero_()
        if keyform_pool is not None:
            _lib.check(lib.cf_rec_build_keyform(dp(keys), n, dp(tab), bbits, fbits, dp(keyform_pool),
                                                dp(self.misc) + 4, self.s._sh()), "cf_rec_build_keyform")
        else:
            _lib.check(lib.cf_rec_build(dp(keys), n, dp(tab), bbits, fbits, dp(self.misc) + 4, self.s._sh()),
                       "cf_rec_build")
        return tab, bbits, fbits

    def _probe(self, launch, maxp: int):
        """Run one probe launch (a function of (pairs, max_pairs)), regrowing the pair
        buffer on overflow; returns (candidate array [k, 2] u64, max_pairs)."""
        while True:
            pairs = self.s._buf("bpairs", maxp * 16)
            self.misc[0].zero_()
            launch(pairs, maxp)
            m = self.misc[:2].cpu().numpy().view(np.uint32)
            npairs, err = int(m[0]), int(m[1])
            if err & _lib.ERR_TABLE_FULL:
                raise _lib.CfError(_lib.CF_EOVERFLOW, "bounded", "join table full (internal error)")
            if err & _lib.ERR_PAIR_OVERFLOW:
                self.misc[1].zero_()
                maxp = max(2 * maxp, npairs + 16)
                continue
            if err:
                raise _lib.CfError(_lib.CF_EBADARG, "bounded", f"record join failed (err {err:#x})")
            pv = pairs[: npairs * 16].cpu().numpy().view(np.uint64).reshape(npairs, 2).copy() if npairs else None
            return pv, maxp

    def join(self, B0, INS, r: int, M: int, P0: int, Icap: int, Dmin: int, split=None, hmax=None):
        """Equal-residue pairs of the filtered sides: D = r-subsets of B0 with prod >= Dmin,
        I = r-subsets of INS with prod < Icap and at most hmax primes above split.
        Returns (pairs as (D index tuple, I index tuple), nD, nI, plan)."""
        inst = _Sides(list(B0), list(INS), r, M, P0)
        return self._join(inst, Icap, Dmin, split, hmax)

    def solve(self, inst, verify: bool = True):
        Icap, Dmin = caps(inst)
        pairs, nD, nI, plan = self._join(inst, Icap, Dmin, None, None)
        return self._finish(inst, pairs, nD, nI, plan, verify)

    def _join(self, inst, Icap, Dmin, split, hmax):
        # the producers launch, fill and upload on the current stream: make it the solver's
        with self.torch.cuda.stream(self.s._torch_stream()):
            return self._join_on_stream(inst, Icap, Dmin, split, hmax)

    NATIVE_MAX_BYTES = 24 << 30     # one-call joins whose workspace would exceed this take the level loop here

    def _join_native(self, inst, Icap, Dmin, split, hmax):
        """The whole instance through cf_bounded_join (one C call: D records, table, I leaves probed,
        candidates back); None when the instance is outside its limits (modulus of 2^64 or more, caps
        of 2^128 or more, a workspace above NATIVE_MAX_BYTES), which the level loop below handles."""
        import ctypes as C
        torch, lib, dp = self.torch, self.lib, _lib.ptr
        r, M = inst.r, inst.M
        B0, INS = list(inst.B0), list(inst.INS)
        if wide_modulus(M) or Icap - 1 >= U128 or Dmin >= U128 or Icap <= 1 or len(B0) < r or len(INS) < r:
            return None
        nb, ni = len(B0), len(INS)
        split_idx = ni if split is None else next((i for i, p in enumerate(INS) if p > split), ni)
        hmax = r if hmax is None else int(hmax)
        if hmax < 0:
            return None
        g = self.gen
        # the instance's four tables (two pool tables, two bound tables) go up in ONE copy: each is
        # built on the host by the library, packed at 256-byte offsets into a page-locked buffer
        parts = [pool_table_host(B0, r, M, 1), pool_table_host(INS, r, M, inst.P0 % M),
                 self._bound_table(lib.cf_ddump_bounds, B0, r, int(Dmin)),
                 self._bound_table(lib.cf_igen_bounds, INS, r, int(Icap))]
        offs, total = [], 0
        for a in parts:
            offs.append(total)
            total += (a.nbytes + 255) // 256 * 256
        if self._stage is None or self._stage.numel() < total:
            self._stage = torch.empty(max(total, 1 << 20), dtype=torch.uint8, pin_memory=True)
        host = self._stage.numpy()
        for o, a in zip(offs, parts):
            host[o:o + a.nbytes] = a.view(np.uint8)
        dev = self.s._buf("bjtab", max(total, 1 << 20))
        with torch.cuda.stream(self.s._torch_stream()):
            dev[:total].copy_(self._stage[:total], non_blocking=True)
        base = dp(dev)
        poolD, poolI, G, H = (base + o for o in offs)
        sh = self.s._sh()
        n_out, need = C.c_uint64(0), C.c_uint64(0)
        sizes = (C.c_uint64 * 2)()
        while True:
            nbytes = self._native_bytes
            tmp = self.s._buf("bjoin", nbytes)
            out = np.zeros(3 * self._native_out, dtype=np.uint64)
            rc = lib.cf_bounded_join(poolD, G, nb, poolI, H, ni, r, M, inst.P0 % M, split_idx, hmax,
                                     0, 0, dp(tmp), nbytes, out.ctypes.data, self._native_out, C.byref(n_out), sizes,
                                     C.byref(need), sh)
            if rc == _lib.CF_ENOMEM:
                grow = max(2 * nbytes, need.value + need.value // 4)
                if grow > self.NATIVE_MAX_BYTES:
                    return None
                self._native_bytes = grow
                continue
            if rc == _lib.CF_EOVERFLOW and n_out.value > self._native_out:
                self._native_out = 2 * n_out.value
                continue
            _lib.check(rc, "cf_bounded_join")
            break
        g.launches += 4 * r + 4
        nD, nI, k = int(sizes[0]), int(sizes[1]), int(n_out.value)
        mo = self._native_out
        did, dkey, iid = out[:k], out[mo:mo + k], out[2 * mo:2 * mo + k]
        if k <= 32:                            # a few candidates (most family instances): no array set-up
            dd_all = [unrank_colex(int(v), r, nb) for v in did]
            ii_all = [unrank_colex(int(v), r, ni) for v in iid]
        else:
            dd_all, ii_all = unrank_colex_batch(did, r, nb).tolist(), unrank_colex_batch(iid, r, ni).tolist()
        pairs = _confirmed_pairs(dd_all, ii_all, dkey, INS, inst.P0 % M, M)
        return pairs, nD, nI, dict(strategy="bounded", Icap=Icap, Dmin=Dmin, table="D", native=True)

    def _bound_table(self, fn, primes, r: int, bound: int) -> np.ndarray:
        """A bound table (cf_ddump_bounds / cf_igen_bounds) of the primes, on the host."""
        n = len(primes)
        nbytes = self.lib.cf_igen_bounds_bytes(n, r)
        out = np.zeros(nbytes, dtype=np.uint8)
        pr = np.asarray(primes, dtype=np.uint64)
        _lib.check(fn(pr.ctypes.data, n, r, bound & (2 ** 64 - 1), bound >> 64, out.ctypes.data, nbytes), "bounds")
        return out

    def _join_on_stream(self, inst, Icap, Dmin, split, hmax):
        if self.native:
            got = self._join_native(inst, Icap, Dmin, split, hmax)
            if got is not None:
                return got
        torch, lib, dp = self.torch, self.lib, _lib.ptr
        r, M = inst.r, inst.M
        plan = dict(strategy="bounded", Icap=Icap, Dmin=Dmin)
        self.misc = self.s._buf("bctr", 64)[:64].view(torch.int32)
        sh = self.s._sh()
        Dk, Did, nD = self.gen.generate_D(inst.B0, r, M, Dmin, bitmask=2)
        poolI, blocks = self.gen.frontiers_I(inst.INS, r, M, inst.P0, Icap, split, hmax)
        blocks = iter(blocks)
        first = next(blocks, None)
        if nD == 0 or first is None:
            nI = sum(b["total"] for b in ([first] if first else []) + list(blocks))
            return [], nD, nI, plan
        second = next(blocks, None)
        maxp = self.s.tuning.pair_capacity
        cands = []                         # (D position, I colex id) arrays
        nI = 0
        if second is None and first["total"] < nD:
            # one small I block: write its leaves and build the table on them
            nI = first["total"]
            plan["table"] = "I"
            if nI:
                Ik = torch.empty(nI, dtype=torch.uint64, device=self.s.device)
                Iid = torch.empty(nI, dtype=torch.uint64, device=self.s.device)
                fr = first
                _lib.check(lib.cf_bgen_expand(0, r - 1, r, len(inst.INS), fr["F"], dp(poolI), dp(fr["key"]),
                                              dp(fr["alo"]), dp(fr["ahi"]), dp(fr["ids"]), dp(fr["meta"]),
                                              dp(fr["offs"]), dp(fr["xs"]), len(inst.INS), 0, 0, nI, dp(Ik), None,
                                              None, dp(Iid), None, sh), "cf_bgen_expand(records)")
                tab, bb, fb = self._table(Ik, nI, plan)
                pv, maxp = self._probe(lambda pairs, mp: _lib.check(
                    lib.cf_rec_probe(dp(Dk), nD, dp(tab), bb, fb, 1, dp(pairs), mp, dp(self.misc),
                                     dp(self.misc) + 4, sh), "cf_rec_probe"), maxp)
                if pv is not None:
                    iid = Iid.view(torch.int64)[torch.from_numpy(pv[:, 1].astype(np.int64)).to(self.s.device)]
                    pv[:, 1] = iid.cpu().numpy().view(np.uint64)
                    cands.append(pv)
        else:
            # the table holds the D records; every I leaf probes it without being written (under the
            # leaves' key form, so that no leaf is converted to a canonical residue; wide moduli write
            # their leaves and probe a table of canonical keys)
            plan["table"] = "D"
            wide = wide_modulus(M)
            tab, bb, fb = self._table(Dk, nD, plan, keyform_pool=None if wide else poolI)
            chain = [first] + ([second] if second is not None else [])
            chunk = self.WIDE_LEAF_CHUNK if wide else self.LEAF_CHUNK
            for fr in _chain(chain, blocks):
                total = fr["total"]
                nI += total
                for c0 in range(0, total, chunk):
                    cc = min(chunk, total - c0)
                    if wide:
                        # the fused leaf probe hashes canonical residues: write the leaves, then probe
                        lb = self.s._buf("bleaf", 16 * cc)
                        Ik, Iid = lb[:8 * cc].view(torch.int64), lb[8 * cc:16 * cc].view(torch.int64)
                        _lib.check(lib.cf_bgen_expand(0, r - 1, r, len(inst.INS), fr["F"], dp(poolI), dp(fr["key"]),
                                                      dp(fr["alo"]), dp(fr["ahi"]), dp(fr["ids"]), dp(fr["meta"]),
                                                      dp(fr["offs"]), dp(fr["xs"]), len(inst.INS), 0, c0, cc,
                                                      dp(Ik), None, None, dp(Iid), None, sh), "cf_bgen_expand(records)")
                        pv, maxp = self._probe(lambda pairs, mp, Ik=Ik, cc=cc: _lib.check(
                            lib.cf_rec_probe(dp(Ik), cc, dp(tab), bb, fb, 0, dp(pairs), mp, dp(self.misc),
                                             dp(self.misc) + 4, sh), "cf_rec_probe"), maxp)
                        if pv is not None:
                            iid = Iid[torch.from_numpy(pv[:, 1].astype(np.int64)).to(self.s.device)]
                            pv[:, 1] = iid.cpu().numpy().view(np.uint64)
                    else:
                        pv, maxp = self._probe(lambda pairs, mp, fr=fr, c0=c0, cc=cc: _lib.check(
                            lib.cf_bgen_probe_keyform(r, len(inst.INS), fr["F"], dp(poolI), dp(fr["key"]),
                                                      dp(fr["ids"]), dp(fr["offs"]), dp(fr["xs"]), c0, cc, dp(tab),
                                                      bb, fb, dp(pairs), mp, dp(self.misc), dp(self.misc) + 4, sh),
                            "cf_bgen_probe_keyform"), maxp)
                    if pv is not None:
                        cands.append(pv)
        pairs = []
        if cands:
            pv = np.concatenate(cands)
            dpos = torch.from_numpy(pv[:, 0].astype(np.int64)).to(self.s.device)
            dk = Dk.view(torch.int64)[dpos].cpu().numpy().view(np.uint64)
            di = Did.view(torch.int64)[dpos].cpu().numpy().view(np.uint64)
            ii_all = unrank_colex_batch(pv[:, 1], r, len(inst.INS))
            dd_all = unrank_colex_batch(di, r, len(inst.B0))
            if wide_modulus(M):                # keys taken mod 2^64: compare the residues themselves
                for dd, ii in zip(map(tuple, dd_all.tolist()), map(tuple, ii_all.tolist())):
                    if (inst.P0 * math.prod(inst.INS[x] for x in ii) - math.prod(inst.B0[x] for x in dd)) % M:
                        continue
                    pairs.append((dd, ii))
            else:
                pairs = _confirmed_pairs(dd_all.tolist(), ii_all.tolist(), dk, inst.INS, inst.P0 % M, M)
        return pairs, nD, nI, plan

    def _finish(self, inst, pairs, nD, nI, plan, verify):
        from .solve import Hit, SolveResult
        r, M = inst.r, inst.M
        hits, pairs_out, above, rejected, screened = [], [], 0, 0, 0
        if pairs:
            B0, INS = inst.B0, inst.INS
            near = log2_screen(inst.P0, B0, INS, pairs, inst.B)
            for (di_, ii_), maybe in zip(pairs, near.tolist()):
                D = tuple(B0[x] for x in di_)
                I = tuple(INS[x] for x in ii_)
                pairs_out.append((D, I))
                if not maybe:                  # log2 n is above log2 B by more than the screen's margin
                    above += 1
                    continue
                dset = set(D)
                fac = tuple(sorted([p for p in B0 if p not in dset] + list(I)))
                n = math.prod(fac)
                if n > inst.B:
                    above += 1
                    continue
                screened += 1
                ok = (n - 1) % M == 0
                if ok and verify:
                    ok, n2, _ = verify_certificate(fac)
                    ok = ok and n2 == n
                if not ok:
                    rejected += 1
                    continue
                hits.append(Hit(D, I, n, fac))
        hits.sort(key=lambda h: (h.n, h.D, h.I))
        pairs_out.sort()
        return SolveResult(hits, nD, nI, len(pairs_out), screened, above, rejected, plan=plan, pairs=pairs_out,
                           launches=self.gen.launches)


def _confirmed_pairs(dd_all, ii_all, dkeys, INS, P0m: int, M: int) -> list:
    """(D index tuple, I index tuple) of every candidate whose residues are equal, P0 * prod(I) == the
    D key (mod M): the table's fingerprint collisions are dropped.  dd_all, ii_all: index rows."""
    pairs = []
    for dd, ii, kd in zip(dd_all, ii_all, np.asarray(dkeys, dtype=np.uint64).tolist()):
        v = P0m
        for x in ii:
            v = v * INS[x] % M
        if v == kd:
            pairs.append((tuple(dd), tuple(ii)))
    return pairs


def log2_screen(P0: int, B0, INS, pairs, bound: int) -> np.ndarray:
    """Which pairs (D index tuple, I index tuple) may have n = P0 * prod(I) / prod(D) at or below
    bound: a float64 screen of log2 n with a margin far above its rounding
    error (sums of at most 32 logarithms of numbers below 2^64), so every pair it rejects is
    certainly above the bound; the pairs it keeps are decided exactly by the caller."""
    if len(pairs) < 64:                        # a few pairs: the exact check alone is cheaper
        return np.ones(len(pairs), dtype=bool)
    dd = np.array([d for d, _ in pairs], dtype=np.int64)
    ii = np.array([i for _, i in pairs], dtype=np.int64)
    lgB = np.log2(np.asarray(B0, dtype=np.float64))
    lgI = np.log2(np.asarray(INS, dtype=np.float64))
    lg = math.log2(P0) - lgB[dd].sum(axis=1) + lgI[ii].sum(axis=1)
    return lg <= math.log2(bound) + 1e-6


class _Sides:
    """The fields of an instance the join needs (base, insertion pool, radius, modulus, P0)."""

    def __init__(self, B0, INS, r, M, P0):
        self.B0, self.INS, self.r, self.M, self.P0 = B0, INS, r, M, P0


def _chain(head, rest):
    yield from head
    yield from rest
