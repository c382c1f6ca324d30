"""solve(M, Q, B0, r, B) -> Carmichael hits: the exchange meet-in-the-middle join on one B200.

A candidate is S = (B0 \\ D) u I with D an r-subset of the base B0 and I an
r-subset of INS = Q \\ B0.  Because every prime q of the pool Q = Q(M) has
(q-1) | M, prod(S) == 1 (mod M) makes S Carmichael by Korselt
(src/mitm64.cpp:12-16).  The congruence is the residue join

    prod(I) == prod(D) * (prod B0)^-1   (mod M)

(the reference matches P0 * prod(I) == prod(D), gpu/mitm_gpu_mstar_driver.py:214-237;
both sides here carry the constant on the D side, so the large I side needs no
multiplier).  Device pipeline, all on one stream:

  1. k_gen_part(D)  : every r-subset of B0, key form, scattered into residue partitions
  2. k_gen_part(I)  : every r-subset of INS (in rank chunks if the side exceeds the budget)
  3. k_join_part    : per partition, shared-memory table of D, stream I, emit equal pairs
  4. k_check_pairs  : recompute residues, fp64 size screen, exact size, Korselt

then one synchronisation, a copy of the (rare) checked pairs, and host
certification of every hit by ``certify.verify_certificate``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .certify import verify_certificate
from .tables import DeviceTables, ncomb, unrank_lex, wide_modulus

RESULT_DTYPE = np.dtype([("flags", "<u4"), ("r", "<u4"), ("d_idx", "<u2", (16,)), ("i_idx", "<u2", (16,))])

# One modulus of the batched kernels (CfBatchMod, cf_batch_mod_bytes() bytes); the
# single-modulus solve uses a one-row array of it for the partitioned table build.
MOD_DTYPE = np.dtype([
    ("poolD", "<u8"), ("tailD", "<u8"), ("poolI", "<u8"), ("tailI", "<u8"), ("screen", "<u8"),
    ("fpw", "<u8"), ("side", "<u8"), ("fill", "<u8"), ("bloom", "<u8"),
    ("nD", "<u8"), ("i_lo", "<u8"), ("nI", "<u8"),
    ("bbits", "<i4"), ("fbits", "<i4"), ("r", "<i4"), ("swap", "<i4"),
    ("pkw", "<u8"), ("psd", "<u8"), ("pcnt", "<u8"), ("pcap", "<u4"), ("plb", "<u4")])


def part_shape(n_build: int, bbits: int, lb: int, sigma: float, max_ranges: int) -> tuple[int, int] | None:
    """(bucket ranges, records per range) of the partitioned table build of n_build
    records into 2^bbits buckets, or None when the table has too many ranges."""
    nparts = 1 << max(0, bbits - lb)
    if nparts > max_ranges:
        return None
    mean = n_build / nparts
    cap = int(math.ceil(mean + sigma * math.sqrt(mean) + 32))
    return nparts, (cap + 3) // 4 * 4
ALL_FLAGS = (_lib.HIT_KEY_EQUAL | _lib.HIT_SCREEN | _lib.HIT_SIZE_EXACT | _lib.HIT_KORSELT | _lib.HIT_DISJOINT)


@dataclass(frozen=True)
class Hit:
    """One Carmichael number found by the join."""
    D: tuple[int, ...]        # deleted base primes (ascending)
    I: tuple[int, ...]        # inserted primes (ascending)
    n: int                    # prod(S)
    factors: tuple[int, ...]  # S, ascending


@dataclass
class SolveResult:
    hits: list[Hit]
    n_D: int                  # D-side records (C(|B0|, r))
    n_I: int                  # I-side records (C(|INS|, r))
    residue_pairs: int        # equal-residue (D, I) pairs (join_sorted's pair count)
    screened: int             # pairs surviving the fp64 log-size screen
    above_bound: int          # equal-residue pairs with prod(S) > B
    rejected: int             # pairs failing the device or host checks (0 unless a bug)
    device_ms: float | None = None
    plan: dict = field(default_factory=dict)
    pairs: list = field(default_factory=list)   # every equal-residue (D primes, I primes) pair
    launches: int = 0                           # kernels of this library launched by the solve

    @property
    def records(self) -> int:
        return self.n_D + self.n_I


@dataclass
class Tuning:
    """Launch shape of the partitioned join (chosen by autotune.py when tuned)."""
    d_per_part: int = 7000          # target D records per partition
    max_pbits: int = 12             # at most 2^12 partitions
    gen_shape: int = 1              # cf_gen_part launch shape (threads x records per thread)
    max_sbits: int = 14             # shared table of 2^sbits slots (4 B) per CTA
    isplit: int = 0                 # CTAs per partition in the join (0 = automatic)
    i_chunk_records: int = 1 << 31  # I-side records per generation/join chunk
    pair_capacity: int = 1 << 14    # initial candidate-pair buffer (grown on overflow)
    sigma: float = 6.0              # partition capacity = mean + sigma*sqrt(mean) + 16
    strategy: str = "fused"         # "fused": table + generate-and-probe; "partition": materialised join;
                                    # "bounded": size-bound-pruned sides + record join; "auto": bounded
                                    # where the bound prunes, else fused
    dtab_load: float = 5.0          # fused: minimum average D records per 16-slot bucket (up to 2x this)
    fused_grid: int = 0             # fused probe CTAs (0 = one per 16384 records)
    l2_table_bytes: int = 72 << 20  # fingerprint arrays above this get a Bloom-filter first level
    max_fbits: int = 21             # Bloom filter at most 2^21 blocks of 32 bytes (64 MB)
    max_nodes: int = 1 << 27        # bounded strategy: frontier nodes per block of first indices
    part_build: bool = True         # fused: partitioned table build for tables of part_min_buckets or more
    part_min_buckets: int = 1 << 21 # smaller tables stay in L2 while built alone: built in place
    part_lb: int = 10               # log2 buckets per range of the partitioned build (9 or 10)
    part_sigma: float = 8.0         # bucket-range capacity = mean + sigma*sqrt(mean) + 32


def dtab_shape(nD: int, tu: Tuning) -> tuple[int, int]:
    """(bbits, fbits) of the D table for nD records: 2^bbits buckets of 16 slots at an
    average load between dtab_load and 2*dtab_load (never above 12), and a Bloom-filter
    first level (about 8 bits per D record, at most 2^max_fbits blocks of 32 bytes) when
    the fingerprint array would not stay in L2 -- and none when that cap leaves fewer than
    6 bits per record."""
    bbits = max(4, int(math.floor(math.log2(max(nD / tu.dtab_load, 2.0)))),
                math.ceil(math.log2(max(nD / 12.0, 2.0))))
    fbits = 0
    if (1 << bbits) * 32 > tu.l2_table_bytes:
        fbits = min(tu.max_fbits, max(4, math.ceil(math.log2(max(nD / 32.0, 2.0)))))
        if (256 << fbits) < 6 * nD:      # under 6 filter bits per record the filter passes nearly everything
            fbits = 0
    return bbits, fbits


def _i_window(inst: "Instance", plan: dict) -> int:
    """Number of I ranks joined: the window [plan["i_lo"], plan["i_limit"]) of [0, C(|INS|, r)), where
    i_lo defaults to 0 and i_limit to C(|INS|, r)."""
    nI = ncomb(len(inst.INS), inst.r)
    lim = plan.get("i_limit")
    hi = nI if lim is None else min(nI, int(lim))
    return max(0, hi - _i_lo(plan))


def _i_lo(plan: dict) -> int:
    """First I rank of the window joined."""
    return int(plan.get("i_lo") or 0)


def _pow2ceil(x: int) -> int:
    return 1 if x <= 1 else 1 << (x - 1).bit_length()


def _cap(mean: float, sigma: float) -> int:
    return int(math.ceil(mean + sigma * math.sqrt(max(mean, 1.0)) + 16))


@dataclass
class Instance:
    M: int
    B0: list[int]
    INS: list[int]
    r: int
    B: int
    P0: int

    @staticmethod
    def build(M: int, Q, B0, r: int, B: int) -> "Instance":
        M, r, B = int(M), int(r), int(B)
        if M < 2 or (M >> ((M & -M).bit_length() - 1)) >= 1 << 63:
            raise ValueError("M must be at least 2 with an odd part below 2^63")
        base = sorted(int(p) for p in B0)
        if len(set(base)) != len(base):
            raise ValueError("B0 has repeated primes")
        bset = set(base)
        ins = sorted(set(int(q) for q in Q) - bset)
        if not (0 <= r <= 10):
            raise ValueError("radius r must be 0..10")
        if len(base) > 1024 or len(ins) > 1024:
            raise ValueError("B0 and Q \\ B0 are limited to 1024 primes each")
        if B < 1:
            raise ValueError("size bound B must be >= 1")
        P0 = math.prod(base)
        if math.gcd(P0 * math.prod(ins), M) != 1:
            raise ValueError("every pool prime must be coprime to M (q does not divide M)")
        if (base and base[-1] >= 1 << 31) or (ins and ins[-1] >= 1 << 31):
            raise ValueError("pool primes must be below 2^31")
        if M % (1 << 33) == 0:
            raise ValueError("2^33 divides M: the solve path needs the 2-adic part of M below 2^33")
        return Instance(M, base, ins, r, B, P0)


def finish_rows(inst: Instance, res: np.ndarray, nD: int, nI: int, plan: dict, verify: bool) -> SolveResult:
    """SolveResult of one modulus from its checked candidate rows (RESULT_DTYPE).

    Rows without CF_HIT_KEY_EQUAL are fingerprint collisions of the fused join and
    are dropped; for the partition join, which compares full keys, they count as
    rejected.  Every hit is re-derived and, with verify, certified on the host."""
    r = inst.r
    hits, screened, above, rejected, pairs = [], 0, 0, 0, []
    bset = inst.B0
    fused = plan.get("strategy") == "fused"
    wide = wide_modulus(inst.M)                # keys taken mod 2^64: confirm every match exactly
    nres = 0
    for row in res:
        f = int(row["flags"])
        if not f & _lib.HIT_KEY_EQUAL:
            if not fused:
                rejected += 1
            continue
        di = [int(x) for x in row["d_idx"][:r]]
        ii = [int(x) for x in row["i_idx"][:r]]
        D = tuple(bset[i] for i in di)
        I = tuple(inst.INS[i] for i in ii)
        if wide and (inst.P0 * math.prod(I) - math.prod(D)) % inst.M:
            if not fused:                     # keys mod 2^64 matched, residues differ
                rejected += 1
            continue
        nres += 1
        pairs.append((D, I))
        if not f & _lib.HIT_SCREEN:
            above += 1
            continue
        screened += 1
        if not f & _lib.HIT_SIZE_EXACT:
            above += 1
            continue
        if (f & ALL_FLAGS) != ALL_FLAGS:
            rejected += 1
            continue
        dset = set(D)
        fac = tuple(sorted([p for p in bset if p not in dset] + list(I)))
        n = 1
        for p in fac:
            n *= p
        ok = n <= inst.B and (n - 1) % inst.M == 0
        if verify and ok:
            ok, n2, _why = verify_certificate(fac)
            ok = ok and n2 == n
        if not ok:
            rejected += 1
            continue
        hits.append(Hit(D, I, n, fac))
    hits.sort(key=lambda x: (x.n, x.D, x.I))
    pairs.sort()
    return SolveResult(hits=hits, n_D=nD, n_I=nI, residue_pairs=nres, screened=screened,
                       above_bound=above, rejected=rejected, plan=dict(plan), pairs=pairs)


class Solver:
    """Reusable device state for repeated solves on one device and stream."""

    def __init__(self, device=None, stream=None, tuning: Tuning | None = None):
        import torch
        self.torch = torch
        self.lib = _lib.load()
        self.device = torch.device(device if device is not None else "cuda")
        if self.device.type != "cuda":
            raise RuntimeError("the join runs on a CUDA device only")
        self.stream = stream
        self.tuning = tuning or Tuning()
        self.tables = DeviceTables(self.device, stream=stream, async_upload=True)
        self._bufs: dict[str, object] = {}
        self._bufset = 0                 # which of two buffer sets the next enqueue uses (solve_many)
        self.d2h_bytes = 0               # bytes read back from the device by collect()
        self._pinned: dict = {}
        self._bounded = None
        self.result_bytes = self.lib.cf_pair_result_bytes()
        assert self.result_bytes == RESULT_DTYPE.itemsize

    # -- buffers -----------------------------------------------------------
    def _buf(self, name: str, nbytes: int):
        key = (name, self._bufset)
        t = self._bufs.get(key)
        if t is None or t.numel() < nbytes:
            t = self.torch.empty(max(nbytes, 16), dtype=self.torch.uint8, device=self.device)
            self._bufs[key] = t
        return t

    def _pinned_buf(self, name: str, nbytes: int):
        """Page-locked host buffer of the current buffer set (rewritten only after the solve that
        last used it has been collected)."""
        key = (name, self._bufset)
        t = self._pinned.get(key)
        if t is None or t.numel() < nbytes:
            t = self.torch.empty(max(nbytes, 64), dtype=self.torch.uint8, pin_memory=True)
            self._pinned[key] = t
        return t

    def _sh(self):
        return _lib.stream_handle(self.stream)

    # -- planning ------------------------------------------------------------
    def plan(self, nD: int, nI: int, capD: int | None = None, capI: int | None = None,
             pairs: int | None = None) -> dict:
        tu = self.tuning
        pbits = min(tu.max_pbits, (_pow2ceil(-(-nD // tu.d_per_part))).bit_length() - 1)
        nparts = 1 << pbits
        chunk = min(nI, tu.i_chunk_records)
        cD = capD or _cap(nD / nparts, tu.sigma)
        cI = capI or _cap(chunk / nparts, tu.sigma)
        cD = min(cD, nD)
        cI = min(cI, chunk) if chunk else 1
        sbits = 4
        while sbits < tu.max_sbits and (1 << (sbits - 1)) < cD:
            sbits += 1
        isplit = tu.isplit or max(1, min(16, (2 * 148 * 2) // max(1, nparts)))
        bbits, fbits = dtab_shape(min(nD, nI), tu)     # the table holds the smaller side
        return dict(pbits=pbits, nparts=nparts, capD=max(cD, 1), capI=max(cI, 1), chunk=max(chunk, 1), sbits=sbits,
                    isplit=isplit, pairs=pairs or tu.pair_capacity, shape=tu.gen_shape, strategy=tu.strategy,
                    bbits=bbits, fbits=fbits, swap=nI < nD)

    # -- one solve -----------------------------------------------------------
    def _mark(self, marks, tag):
        if marks is not None:
            ev = self.torch.cuda.Event(enable_timing=True)
            ev.record(self._torch_stream())
            marks.append((tag, ev))

    def enqueue(self, inst: Instance, plan: dict, marks: list | None = None):
        """Queue the whole device pipeline for `inst` on the stream (no host sync).
        `marks` (optional list) receives (tag, CUDA event) pairs around every kernel."""
        if plan.get("strategy", "fused") == "fused":
            return self._enqueue_fused(inst, plan, marks)
        return self._enqueue_partition(inst, plan, marks)

    def _side_tables(self, inst: Instance, side: str):
        """(pool, tail) device tables of one side: D with multiplier (prod B0)^-1, I with 1."""
        M, r = inst.M, inst.r
        primes, mult = (inst.B0, pow(inst.P0, -1, M)) if side == "D" else (inst.INS, 1)
        pool = self.tables.pool(primes, r, M, mult)
        return pool, self.tables.tail(primes, r, M, mult, pool)

    def _tables_for(self, inst: Instance):
        poolD, tailD = self._side_tables(inst, "D")
        poolI, tailI = self._side_tables(inst, "I")
        screen = self.tables.screen(inst.P0, inst.B, 1e-6)
        return poolD, poolI, tailD, tailI, screen

    def _enqueue_fused(self, inst: Instance, plan: dict, marks: list | None):
        """D table build, fused generate-and-probe of the I side, pair check."""
        torch, lib = self.torch, self.lib
        r = inst.r
        nD, nIt = ncomb(len(inst.B0), r), _i_window(inst, plan)
        bbits, fbits = plan["bbits"], plan.get("fbits", 0)
        tbytes = lib.cf_dtab_bytes2(bbits, fbits)
        tab = self._buf("dtab", tbytes)
        ctr = self._buf("ctr", 64)
        misc = ctr[:64].view(torch.int32)
        maxp = plan["pairs"]
        pairs = self._buf("pairs", maxp * 16)
        res = self._buf("res", maxp * self.result_bytes)
        sh = self._sh()
        dp = _lib.ptr
        ck = _lib.check
        misc.zero_()
        nb = 1 << bbits
        tab[: 32 * nb].zero_()                     # fingerprint sectors
        tab[160 * nb: tbytes].zero_()              # fill counters and Bloom filter
        # build on the smaller side (swap: the table holds the I window and the D side probes)
        swap = bool(plan.get("swap")) and nIt < nD
        bside, pside = ("I", "D") if swap else ("D", "I")
        bn, bcount = (len(inst.INS), nIt) if swap else (len(inst.B0), nD)
        pn, pcount = (len(inst.B0), nD) if swap else (len(inst.INS), nIt)
        tu = self.tuning
        pshape = None
        if tu.part_build and not plan.get("no_part") and nb >= tu.part_min_buckets and r <= lib.cf_batch_max_r():
            pshape = part_shape(bcount, bbits, tu.part_lb, tu.part_sigma, lib.cf_batch_part_max_ranges())
        # in-place builds of tables of at most 2^20 buckets use compact side words (half the side area,
        # L2-resident while built); partitioned builds and larger tables the wide entries
        side_format = 1 if pshape is None and bbits <= 20 else 0
        self._mark(marks, "start")
        ilo = _i_lo(plan)                          # first I rank of the window
        if pshape is not None:
            tables = self._tables_for(inst)
            self._part_build(inst, plan, pshape, tables, tab, nD, nIt, swap, misc)
            poolD, poolI, tailD, tailI, screen = tables
            ppool, ptail = (poolD, tailD) if pside == "D" else (poolI, tailI)
        else:
            # the build side's tables first: the table build runs while the host prepares the other side
            bpool, btail = self._side_tables(inst, bside)
            ck(lib.cf_dtab_build3(dp(bpool), dp(btail), bn, r, ilo if swap else 0, bcount, dp(tab), bbits, fbits,
                                  side_format, dp(misc) + 4, sh), "cf_dtab_build")
            ppool, ptail = self._side_tables(inst, pside)
            screen = self.tables.screen(inst.P0, inst.B, 1e-6)
            poolD, poolI = (bpool, ppool) if bside == "D" else (ppool, bpool)
        ppool, ptail = dp(ppool), dp(ptail)
        self._mark(marks, "gen_D")
        ck(lib.cf_fused_probe3(ppool, ptail, pn, r, 0 if swap else ilo, pcount, dp(tab), bbits, fbits, side_format,
                               ilo if swap else 0, int(swap), dp(pairs), maxp, dp(misc), dp(misc) + 4,
                               self.tuning.fused_grid, sh), "cf_fused_probe")
        self._mark(marks, "probe")
        ck(lib.cf_check_pairs(dp(poolD), dp(poolI), dp(screen), r, dp(pairs), dp(misc), maxp, dp(res),
                              dp(misc) + 4, sh), "cf_check_pairs")
        self._mark(marks, "check")
        return dict(misc=misc, dcnt=None, icnt=None, res=res, nD=nD, nI=nIt, plan=plan, launches=3)

    def _part_build(self, inst: Instance, plan: dict, pshape: tuple, tables: tuple, tab, nD: int, nIt: int,
                    swap: bool, misc):
        """Partitioned table build (scatter by bucket range, shared-memory range build,
        overflow fix-up) through a one-modulus descriptor of the batched kernels."""
        torch, lib = self.torch, self.lib
        dp, ck, sh = _lib.ptr, _lib.check, self._sh()
        poolD, poolI, tailD, tailI, screen = tables
        bbits, fbits = plan["bbits"], plan.get("fbits", 0)
        nb = 1 << bbits
        nparts, cap = pshape
        n_build = nIt if swap else nD
        tile = lib.cf_batch_part_tile()
        # scratch: range counters, then the records of every range (4 + 8 bytes each)
        ocap = 1 << 12
        obytes = ocap * lib.cf_batch_ovf_bytes()
        up = lambda x: (x + 255) // 256 * 256
        scr = self._buf("pscratch", up(nparts * 4) + up(64) + up(obytes) + up(nparts * cap * 4) + nparts * cap * 8)
        base = dp(scr)
        pcnt, pmisc = base, base + up(nparts * 4)
        ovf = pmisc + up(64)
        pkw = ovf + up(obytes)
        psd = pkw + up(nparts * cap * 4)
        row = np.zeros(1, dtype=MOD_DTYPE)
        row["poolD"], row["tailD"], row["poolI"], row["tailI"] = dp(poolD), dp(tailD), dp(poolI), dp(tailI)
        row["screen"] = dp(screen)
        t0 = dp(tab)
        row["fpw"], row["side"], row["fill"] = t0, t0 + 32 * nb, t0 + 160 * nb
        row["bloom"] = t0 + 164 * nb if fbits else 0
        row["nD"], row["i_lo"], row["nI"] = nD, _i_lo(plan), nIt
        row["bbits"], row["fbits"], row["r"], row["swap"] = bbits, fbits, inst.r, int(swap)
        row["pkw"], row["psd"], row["pcnt"], row["pcap"], row["plb"] = pkw, psd, pcnt, cap, self.tuning.part_lb
        host = np.zeros(MOD_DTYPE.itemsize // 8 + 4, dtype=np.uint64)
        host[: MOD_DTYPE.itemsize // 8] = row.view(np.uint64)
        k = MOD_DTYPE.itemsize // 8
        host[k:k + 4] = (0, -(-n_build // tile), 0, nparts)        # scatter and range ticket prefix sums
        # pinned staging of this buffer set, rewritten only after its previous solve has been collected
        stage = self._pinned_buf("pdesc", host.nbytes)
        stage[: host.nbytes].numpy()[:] = host.view(np.uint8)
        hdev = self._buf("pdesc", host.nbytes)
        with torch.cuda.stream(self._torch_stream()):
            hdev[: host.nbytes].copy_(stage[: host.nbytes], non_blocking=True)
        self.h2d_desc_bytes = getattr(self, "h2d_desc_bytes", 0) + host.nbytes
        mods, tsS, tsP = dp(hdev), dp(hdev) + 8 * k, dp(hdev) + 8 * k + 16
        scr[: up(nparts * 4) + 64].zero_()
        err = dp(misc) + 4
        lb = self.tuning.part_lb
        ck(lib.cf_batch_part(0, mods, tsS, 1, pmisc, None, 0, pmisc + 24, err, lb, inst.r, 0, sh),
           "cf_batch_part(scatter)")
        ck(lib.cf_batch_part(1, mods, tsP, 1, pmisc + 8, ovf, ocap, pmisc + 24, err, lb, 0, 0, sh),
           "cf_batch_part(place)")
        ck(lib.cf_batch_part(2, mods, None, 1, None, ovf, ocap, pmisc + 24, err, lb, 0, 0, sh), "cf_batch_part(fix)")

    def _enqueue_partition(self, inst: Instance, plan: dict, marks: list | None):
        """Partitioned generation of both sides and the shared-memory partition join."""
        torch, lib = self.torch, self.lib
        r, M = inst.r, inst.M
        nD, nIt = ncomb(len(inst.B0), r), _i_window(inst, plan)
        P = plan["nparts"]
        pbits, shape = plan["pbits"], plan["shape"]
        multD = pow(inst.P0, -1, M)
        poolD = self.tables.pool(inst.B0, r, M, multD)
        poolI = self.tables.pool(inst.INS, r, M, 1)
        tailD = self.tables.tail(inst.B0, r, M, multD, poolD)
        tailI = self.tables.tail(inst.INS, r, M, 1, poolI)
        screen = self.tables.screen(inst.P0, inst.B, 1e-6)
        capD, capI, chunk = plan["capD"], plan["capI"], plan["chunk"]
        Dbuf = self._buf("D", P * capD * 16)
        Ibuf = self._buf("I", P * capI * 16)
        ctr = self._buf("ctr", (2 * P + 8) * 4)
        ctr_u32 = ctr[: (2 * P + 8) * 4].view(torch.int32)
        dcnt = ctr_u32[:P]
        icnt = ctr_u32[P:2 * P]
        misc = ctr_u32[2 * P:]          # [0] npairs, [1] err
        maxp = plan["pairs"]
        pairs = self._buf("pairs", maxp * 16)
        res = self._buf("res", maxp * self.result_bytes)
        sh = self._sh()
        dp = _lib.ptr
        ctr_u32.zero_()
        ck = _lib.check
        launches = 0
        self._mark(marks, "start")
        ck(lib.cf_gen_part(dp(poolD), dp(tailD), len(inst.B0), r, 0, nD, pbits, capD, dp(dcnt), dp(Dbuf),
                           dp(misc) + 4, shape, sh), "cf_gen_part(D)")
        launches += 1
        self._mark(marks, "gen_D")
        ilo = _i_lo(plan)
        for off in range(0, nIt, chunk):
            cnt = min(chunk, nIt - off)
            lo = ilo + off
            if off:
                icnt.zero_()
            ck(lib.cf_gen_part(dp(poolI), dp(tailI), len(inst.INS), r, lo, cnt, pbits, capI, dp(icnt), dp(Ibuf),
                               dp(misc) + 4, shape, sh), "cf_gen_part(I)")
            self._mark(marks, "gen_I")
            ck(lib.cf_join_part(dp(Dbuf), dp(dcnt), capD, dp(Ibuf), dp(icnt), capI, pbits, plan["sbits"],
                                plan["isplit"], 0, dp(pairs), maxp, dp(misc), dp(misc) + 4, sh),
               "cf_join_part")
            self._mark(marks, "join")
            launches += 2
        ck(lib.cf_check_pairs(dp(poolD), dp(poolI), dp(screen), r, dp(pairs), dp(misc), maxp, dp(res),
                              dp(misc) + 4, sh), "cf_check_pairs")
        launches += 1
        self._mark(marks, "check")
        return dict(misc=misc, dcnt=dcnt, icnt=icnt, res=res, nD=nD, nI=nIt, plan=plan, launches=launches)

    def collect(self, inst: Instance, h: dict, verify: bool = True) -> tuple[SolveResult | None, dict | None]:
        """Synchronise, read counters; returns (result, None) or (None, bigger plan) on overflow."""
        ev = h.get("ev")
        if ev is None:
            self._torch_stream().synchronize()
            misc = h["misc"][:2].cpu().numpy().view(np.uint32)
            self.d2h_bytes += 8
        else:                                      # staged by _stage_readback: wait for this solve only
            ev.synchronize()
            misc = h["hread"][:8].numpy().view(np.uint32).copy()
            self.d2h_bytes += 8 + h["hrows"] * self.result_bytes
        npairs, err = int(misc[0]), int(misc[1])
        plan = h["plan"]
        if err & _lib.ERR_TABLE_FULL:
            raise _lib.CfError(_lib.CF_EOVERFLOW, "solve", "D table full (internal error)")
        if err & (_lib.ERR_PART_OVERFLOW | _lib.ERR_PAIR_OVERFLOW):
            newp = dict(plan)
            if err & _lib.ERR_PART_OVERFLOW and h["dcnt"] is None:
                newp["no_part"] = True          # fused: a bucket range of the table build overflowed
            elif err & _lib.ERR_PART_OVERFLOW:
                dmax = int(h["dcnt"].max().item())
                imax = int(h["icnt"].max().item())
                newp["capD"] = max(plan["capD"], dmax + 16)
                newp["capI"] = max(plan["capI"], imax + 16)
            if err & _lib.ERR_PAIR_OVERFLOW:
                newp["pairs"] = max(plan["pairs"] * 2, npairs + 16)
            return None, newp
        if err & _lib.ERR_SPIN_LIMIT:
            raise _lib.CfError(_lib.CF_ETIMEOUT, "solve", "a bounded device wait gave up")
        if err & 32:
            raise _lib.CfError(_lib.CF_EBADARG, "solve", "a kernel rejected its arguments (pool primes >= 2^31?)")
        if err & _lib.ERR_KEY_MISMATCH:
            raise _lib.CfError(_lib.CF_EBADARG, "solve", "checked pair with unequal residues (internal error)")
        nb = npairs * self.result_bytes
        if ev is not None and npairs <= h["hrows"]:
            res = np.frombuffer(h["hread"][8:8 + nb].numpy().tobytes(), dtype=RESULT_DTYPE)
        else:
            res = np.frombuffer(h["res"][:nb].cpu().numpy().tobytes(), dtype=RESULT_DTYPE)
            self.d2h_bytes += nb
        return self._finish(inst, h, res, verify), None

    def _finish(self, inst: Instance, h: dict, res: np.ndarray, verify: bool) -> SolveResult:
        return finish_rows(inst, res, h["nD"], h["nI"], h["plan"], verify)

    def _direct_plan(self, inst: Instance, i_limit: int | None, i_lo: int = 0) -> dict | None:
        """The device plan of a fused or partition join of inst over the I ranks [i_lo, i_limit), or
        None when inst takes another path (radius 0, the bounded strategy, an empty window)."""
        if inst.r == 0:
            return None
        st = self.tuning.strategy
        if i_limit is None and not i_lo and (st == "bounded" or st == "auto"):
            from . import bsolve
            if bsolve.applicable(inst) and (st == "bounded" or bsolve.prunes(inst)):
                return None
        nD = ncomb(len(inst.B0), inst.r)
        nI = _i_window(inst, {"i_limit": i_limit, "i_lo": i_lo})
        if nI == 0 or nD == 0:
            return None
        plan = self.plan(nD, nI)
        plan["i_limit"] = i_limit
        plan["i_lo"] = int(i_lo)
        if min(nD, nI) >= 1 << 32:        # ranks in the fused table are 32-bit
            plan["strategy"] = "partition"
        return plan

    def _replan(self, inst: Instance, newp: dict) -> dict:
        """The plan after an overflow: the capacities collect() asked for."""
        nD, nI = ncomb(len(inst.B0), inst.r), _i_window(inst, newp)
        plan = self.plan(nD, nI, newp["capD"], newp["capI"], newp["pairs"])
        plan["strategy"] = newp.get("strategy", plan["strategy"])
        plan["i_limit"] = newp.get("i_limit")
        plan["i_lo"] = _i_lo(newp)
        plan["no_part"] = newp.get("no_part", False)
        return plan

    def solve_instance(self, inst: Instance, verify: bool = True, timed: bool = False,
                       marks: list | None = None, i_limit: int | None = None, i_lo: int = 0) -> SolveResult:
        """Join one instance.  i_lo, i_limit: join only the I ranks [i_lo, i_limit) (a bounded
        sample of the instance, or one device's share of it; every pair with such an I rank
        is found).  n_I of the result is the window's size."""
        if i_lo < 0 or (i_limit is not None and i_limit < 0):
            raise ValueError("the I-rank window must not start or end below 0")
        plan = self._direct_plan(inst, i_limit, i_lo)
        if plan is None:
            if inst.r == 0:
                return self._solve_r0(inst)
            st = self.tuning.strategy
            if i_limit is None and not i_lo and (st == "bounded" or st == "auto"):
                from . import bsolve
                if bsolve.applicable(inst) and (st == "bounded" or bsolve.prunes(inst)):
                    if self._bounded is None:
                        self._bounded = bsolve.BoundedSolve(self)
                    return self._bounded.solve(inst, verify)
            nD = ncomb(len(inst.B0), inst.r)
            return SolveResult([], nD, _i_window(inst, {"i_limit": i_limit, "i_lo": i_lo}), 0, 0, 0, 0)
        return self._run_plan(inst, plan, verify, timed, marks)

    def _run_plan(self, inst: Instance, plan: dict, verify: bool, timed: bool = False,
                  marks: list | None = None) -> SolveResult:
        """Enqueue, collect, and re-run with larger capacities while a buffer overflows."""
        for _attempt in range(6):
            ev0 = ev1 = None
            if timed:
                ev0 = self.torch.cuda.Event(enable_timing=True)
                ev1 = self.torch.cuda.Event(enable_timing=True)
                ev0.record(self._torch_stream())
            if marks is not None:
                marks.clear()
            h = self.enqueue(inst, plan, marks)
            if timed:
                ev1.record(self._torch_stream())
            out, newp = self.collect(inst, h, verify)
            if out is not None:
                if timed:
                    out.device_ms = ev0.elapsed_time(ev1)
                out.launches = h["launches"]
                return out
            plan = self._replan(inst, newp)
        raise _lib.CfError(_lib.CF_EOVERFLOW, "solve", "capacities kept overflowing")

    def _stage_readback(self, h: dict, rows: int):
        """Queue, behind a solve's kernels, the copy of its counters and of its first `rows`
        checked rows into page-locked memory, and an event after them: collect() then waits
        for this solve alone, not for work queued after it."""
        torch = self.torch
        rb = self.result_bytes
        rows = max(0, min(int(rows), int(h["plan"]["pairs"])))
        hm = self._pinned_buf("readback", 8 + rows * rb)
        st = self._torch_stream()
        with torch.cuda.stream(st):
            hm[:8].copy_(h["misc"][:2].view(torch.uint8), non_blocking=True)
            if rows:
                hm[8:8 + rows * rb].copy_(h["res"][: rows * rb], non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(st)
        h.update(ev=ev, hread=hm, hrows=rows)

    def solve_many(self, insts: list, verify: bool = True, marks_list: list | None = None,
                   i_limit: int | None = None, readback_rows: int = 256, streams: int = 2,
                   i_lo: int = 0) -> list[SolveResult]:
        """Solve instances one after another, each with its own build, probe and check, while
        the host collects and certifies each one as the device runs the next: two buffer sets
        alternate, and every solve's counters and first checked rows come back behind its own
        kernels.  With streams = 2 the two buffer sets also have a CUDA stream each, so one
        solve's table build can run beside the previous solve's probe.  The results equal
        solve_instance's on each instance (i_lo, i_limit: the same I-rank window for every
        instance).  marks_list (optional list) receives one marks list per instance (see
        enqueue)."""
        torch = self.torch
        out: list = [None] * len(insts)
        base = self._torch_stream()
        saved = (self.stream, self.tables.stream)
        if getattr(self, "_many_streams", None) is None:
            self._many_streams = [torch.cuda.Stream(self.device), torch.cuda.Stream(self.device)]
        sts = self._many_streams[:2] if streams > 1 else [base]
        for st in sts:
            if st is not base:
                st.wait_stream(base)               # after everything queued before the call

        def use(k):
            self._bufset = k & 1
            st = sts[k & 1] if len(sts) > 1 else sts[0]
            self.stream = st
            self.tables.stream = st
            return torch.cuda.stream(st)

        pending = None
        try:
            for i in range(len(insts) + 1):
                cur = None
                if i < len(insts):
                    inst = insts[i]
                    marks = None
                    if marks_list is not None:
                        marks = []
                        marks_list.append(marks)
                    with use(i):                   # the set (and stream) the solve in flight does not use
                        plan = self._direct_plan(inst, i_limit, i_lo)
                        if plan is None:
                            out[i] = self.solve_instance(inst, verify=verify, marks=marks, i_limit=i_limit,
                                                         i_lo=i_lo)
                        else:
                            h = self.enqueue(inst, plan, marks)
                            self._stage_readback(h, readback_rows)
                            cur = (i, h, marks)
                if pending is not None:
                    j, h, marks = pending
                    with use(j):
                        res, newp = self.collect(insts[j], h, verify)
                        if res is None:            # an overflow: run it again alone, larger
                            res = self._run_plan(insts[j], self._replan(insts[j], newp), verify, marks=marks)
                        else:
                            res.launches = h["launches"]
                    out[j] = res
                pending = cur
        finally:
            self._bufset = 0
            self.stream, self.tables.stream = saved
            for st in sts:
                if st is not base:
                    base.wait_stream(st)           # work queued after the call follows every solve
        return out

    def _torch_stream(self):
        return self.stream if self.stream is not None else self.torch.cuda.current_stream(self.device)

    def _solve_r0(self, inst: Instance) -> SolveResult:
        n = inst.P0
        hits = []
        if n % inst.M == 1 % inst.M and n <= inst.B:
            ok, _, _ = verify_certificate(inst.B0)
            if ok:
                hits.append(Hit((), (), n, tuple(inst.B0)))
        return SolveResult(hits, 1, 1, int(n % inst.M == 1 % inst.M), len(hits), 0, 0)

    def solve(self, M: int, Q, B0, r: int, B: int, verify: bool = True, timed: bool = False) -> SolveResult:
        return self.solve_instance(Instance.build(M, Q, B0, r, B), verify=verify, timed=timed)


_default_solvers: dict = {}


def solve(M: int, Q, B0, r: int, B: int, device=None, verify: bool = True, strategy: str = "fused") -> SolveResult:
    """Every Carmichael hit S = (B0 \\ D) u I with |D| = |I| = r, prod(S) == 1 (mod M), prod(S) <= B.

    Q is the eligible pool Q(M) (primes q with (q-1) | M and q not dividing M);
    INS = Q \\ B0.  Hits are certified on the host and returned ascending by n.
    strategy: "fused" (table + generate-and-probe), "partition" (materialised join), "bounded"
    (both sides pruned by the size bound, then a record join) or "auto" (bounded where the
    bound prunes, else fused).  Every strategy returns the same hits."""
    import torch
    dev = torch.device(device if device is not None else "cuda")
    key = (dev.type, dev.index, strategy)
    s = _default_solvers.get(key)
    if s is None:
        s = _default_solvers[key] = Solver(dev, tuning=Tuning(strategy=strategy))
    return s.solve(M, Q, B0, r, B, verify=verify)


def solve_many(instances, device=None, verify: bool = True, strategy: str = "fused") -> list[SolveResult]:
    """solve() over a list of (M, Q, B0, r, B) tuples (or objects with those attributes), in order:
    each instance is joined on its own on the device, while the host prepares the next one's
    tables and collects and certifies the previous one.  Returns one SolveResult per instance,
    equal to solve()'s."""
    import torch
    dev = torch.device(device if device is not None else "cuda")
    key = (dev.type, dev.index, strategy)
    s = _default_solvers.get(key)
    if s is None:
        s = _default_solvers[key] = Solver(dev, tuning=Tuning(strategy=strategy))
    xs = []
    for w in instances:
        M, Q, B0, r, B = (w.M, w.Q, w.B0, w.r, w.B) if hasattr(w, "M") else w
        xs.append(Instance.build(M, Q, B0, r, B))
    return s.solve_many(xs, verify=verify)


def decode_pair(inst: Instance, d_rank: int, i_rank: int):
    """(D primes, I primes) of a pair of lexicographic ranks."""
    di = unrank_lex(d_rank, len(inst.B0), inst.r)
    ii = unrank_lex(i_rank, len(inst.INS), inst.r)
    return tuple(inst.B0[i] for i in di), tuple(inst.INS[i] for i in ii)
