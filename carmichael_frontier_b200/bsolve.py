"""Product-bounded solve: prune both sides by the size bound before the join.

A hit S = (B0 \\ D) u I needs prod(S) = P0 * prod(I) / prod(D) <= B.  With
Dmax = the product of the r largest base primes and Imin = the product of the r
smallest insertion primes this gives the reference driver's two filters
(gpu/mitm_gpu_mstar_driver.py:189-203, with U = B + 1):

    prod(I) <  Icap = min(prod of the r largest INS + 1, floor(B * Dmax / P0) + 1)
    prod(D) >= Dmin = ceil(P0 * Imin / B)

The filtered sides come from the bounded producers (csrc/cf_bgen.cu: the igen /
idump and ddump records), are joined by the record hash join (csrc/cf_rec_join.cu,
table on the smaller side), and every equal-key pair is checked exactly on the
host (prod(S) <= B, prod(S) == 1 mod M, certificate), as run_instance does
(:241-262).  The hit set equals the unpruned join's: pruning removes only
subsets that no hit can contain.  Where the bound prunes hard (B = prod(B0) *
10^4, the serving workload) the sides are a tiny fraction of C(n, r).
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib
from .bounded import U128, _cat_u64
from .certify import verify_certificate
from .tables import unrank_colex

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


def prunes(inst) -> bool:
    """True when the bound removes part of either side (else the fused join is cheaper)."""
    r = inst.r
    Icap, Dmin = caps(inst)
    return Icap <= math.prod(inst.INS[-r:]) or Dmin > math.prod(inst.B0[:r])


class BoundedSolve:
    """Solves one instance with the bounded producers and the record hash join."""

    def __init__(self, solver):
        from .bounded import BoundedGenerator
        self.s = solver
        self.torch = solver.torch
        self.lib = solver.lib
        self.gen = BoundedGenerator(solver.device)

    def generate(self, inst, i_chunk: int = 1 << 28):
        """Filtered sides on the device: (Dk, Did, [(Ik, Iid), ...], nD, nI, caps)."""
        Icap, Dmin = caps(inst)
        Dk, Did, nD = self.gen.generate_D(inst.B0, inst.r, inst.M, Dmin, bitmask=2)
        chunks = list(self.gen.generate_I(inst.INS, inst.r, inst.M, inst.P0, Icap, max_records=i_chunk))
        nI = sum(int(k.numel()) for k, _ in chunks)
        return Dk, Did, chunks, nD, nI, (Icap, Dmin)

    def solve(self, inst, verify: bool = True):
        from .solve import Hit, SolveResult, dtab_shape
        torch, lib, dp, ck = self.torch, self.lib, _lib.ptr, _lib.check
        r = inst.r
        Dk, Did, chunks, nD, nI, (Icap, Dmin) = self.generate(inst)
        plan = dict(strategy="bounded", Icap=Icap, Dmin=Dmin)
        if nD == 0 or nI == 0:
            return SolveResult([], nD, nI, 0, 0, 0, 0, plan=plan)
        # the table holds the smaller side (the I side only when it is one chunk)
        swap = len(chunks) == 1 and nI < nD
        if (nI if swap else nD) >= RANK_LIMIT:
            raise _lib.CfError(_lib.CF_EOVERFLOW, "bounded", "table side has 2^32 records or more")
        build = chunks[0][0] if swap else Dk
        nb = nI if swap else nD
        bbits, fbits = dtab_shape(nb, self.s.tuning)
        plan.update(bbits=bbits, fbits=fbits, swap=swap)
        tbytes = lib.cf_dtab_bytes2(bbits, fbits)
        tab = self.s._buf("btab", tbytes)
        ctr = self.s._buf("bctr", 64)
        misc = ctr[:64].view(torch.int32)
        sh = self.s._sh()
        nbk = 1 << bbits
        tab[: 32 * nbk].zero_()
        tab[160 * nbk: tbytes].zero_()
        misc.zero_()
        ck(lib.cf_rec_build(dp(build), nb, dp(tab), bbits, fbits, dp(misc) + 4, sh), "cf_rec_build")
        probes = [(Dk, 0)] if swap else []
        if not swap:
            off = 0
            for k, _ in chunks:
                probes.append((k, off))
                off += int(k.numel())
        maxp = self.s.tuning.pair_capacity
        found = []
        for keys, off in probes:
            while True:
                pairs = self.s._buf("bpairs", maxp * 16)
                misc[0].zero_()
                ck(lib.cf_rec_probe(dp(keys), keys.numel(), dp(tab), bbits, fbits, int(swap), dp(pairs), maxp,
                                    dp(misc), dp(misc) + 4, sh), "cf_rec_probe")
                m = misc[:2].cpu().numpy().view(np.uint32)
                npairs, err = int(m[0]), int(m[1])
                if err & _lib.ERR_TABLE_FULL:
                    raise _lib.CfError(_lib.CF_EOVERFLOW, "bounded", "join table full (internal error)")
                if err & _lib.ERR_PAIR_OVERFLOW:
                    misc[1].zero_()
                    maxp = max(2 * maxp, npairs + 16)
                    continue
                if err:
                    raise _lib.CfError(_lib.CF_EBADARG, "bounded", f"record join failed (err {err:#x})")
                if npairs:
                    pv = pairs[: npairs * 16].cpu().numpy().view(np.uint64).reshape(npairs, 2).copy()
                    pv[:, 1] += np.uint64(off)        # I positions of a probing chunk start at its offset
                    found.append(pv)
                break
        Ik_all = _cat_u64([k for k, _ in chunks])
        Iid_all = _cat_u64([i for _, i in chunks])
        hits, pairs_out, above, rejected, screened = [], [], 0, 0, 0
        if found:
            pv = np.concatenate(found)
            dpos = torch.from_numpy(pv[:, 0].astype(np.int64)).to(self.s.device)
            ipos = torch.from_numpy(pv[:, 1].astype(np.int64)).to(self.s.device)
            dk = Dk.view(torch.int64)[dpos].cpu().numpy().view(np.uint64)
            ik = Ik_all.view(torch.int64)[ipos].cpu().numpy().view(np.uint64)
            di = Did.view(torch.int64)[dpos].cpu().numpy().view(np.uint64)
            ii = Iid_all.view(torch.int64)[ipos].cpu().numpy().view(np.uint64)
            B0, INS = inst.B0, inst.INS
            for j in np.nonzero(dk == ik)[0]:
                D = tuple(B0[x] for x in unrank_colex(int(di[j]), r, len(B0)))
                I = tuple(INS[x] for x in unrank_colex(int(ii[j]), r, len(INS)))
                pairs_out.append((D, I))
                dset = set(D)
                fac = tuple(sorted([p for p in B0 if p not in dset] + list(I)))
                n = math.prod(fac)
                if n > inst.B:
                    above += 1
                    continue
                screened += 1
                ok = (n - 1) % inst.M == 0
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
