"""Batched portfolio: many moduli (uneven pool sizes, mixed radii) in persistent kernels.

The reference solves one instance at a time: ``run_instance``
(gpu/mitm_gpu_mstar_driver.py:184-286) generates, sorts and joins each side with
the CuPy kernels of gpu/mitm_gpu2.py and is called per instance from the driver
loop (:311).  Here a whole portfolio is split into batches whose tables fit a
memory budget, and each batch is four device operations on one stream:

  zero   the fingerprint arrays, fill counters and Bloom filters of the batch
  k_batch<0>     every modulus's table from its smaller side   (persistent, device work queue)
  k_batch<1>     probes of every table by the other side       (persistent, device work queue)
  k_batch_check  every candidate pair, any radius

followed by one synchronisation and host certification of the hits.  Tickets of
the work queue are ordered by modulus, so the table being probed stays in L2
while a modulus is worked on, and small moduli cost no launch of their own.
The per-batch sequence is fixed, so ``run(..., graphs=True)`` captures it once
per batch in a CUDA graph and replays it.

Two per-modulus forms are kept for comparison:
  run_plain        the reference's form on this GPU: mitm_gpu2 generate ->
                   sort_side -> join_sorted per modulus (one modulus per launch
                   sequence), host exact check of the pairs
  run_per_modulus  this library's single-modulus fused solve, one modulus at a time
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .certify import verify_certificate
from .solve import (MOD_DTYPE, RESULT_DTYPE, Hit, Instance, SolveResult, Solver, Tuning, dtab_shape, finish_rows,
                    part_shape)
from .tables import ncomb, pool_table_host, screen_table_host

_ALIGN = 256


def _up(x: int, a: int = _ALIGN) -> int:
    return (x + a - 1) // a * a


def tu_ovf_bytes(solver) -> int:
    """Bytes of the overflow list of the partitioned build."""
    return max(64, solver.tuning.ovf_capacity * solver.lib.cf_batch_ovf_bytes())


@dataclass
class BatchTuning:
    """Launch shape of the batched kernels (chosen by autotune.tune_batch when tuned)."""
    ticket: int = 4096                 # records per work-queue ticket (multiple of 32; tune_batch's pick on
                                       # the 1024-modulus portfolio: 512 ms against 520 / 529 / 566 ms at
                                       # 2048 / 8192 / 16384)
    grid: int = 0                      # persistent CTAs per launch (0 = one resident wave)
    mem_budget: int = 24 << 30         # D-table bytes of one batch
    pair_capacity: int = 1 << 16       # initial candidate buffer (grown on overflow)
    dtab: Tuning = field(default_factory=Tuning)   # D-table sizing (dtab_load, Bloom level)
    part_build: bool = True            # partitioned table build for tables above part_min_buckets
    part_min_buckets: int = 1 << 16    # smaller tables (L2-resident) are built in place
    part_lb: int = 10                  # log2 buckets per range of the partitioned build (9 or 10)
    part_sigma: float = 8.0            # bucket-range capacity = mean + sigma*sqrt(mean) + 32
    ovf_capacity: int = 1 << 16        # records that ran past their bucket range (per batch)
    probe_per_radius: bool = True      # one probe launch per radius (kernels carry one radius's code)
    overlap: bool = True               # consecutive batches alternate between two arenas and streams


@dataclass
class _Batch:
    idx: list                          # portfolio positions of the moduli in this batch
    mods: object = None                # device CfBatchMod[nmod]
    tsD: object = None                 # device u64[nmod+1] ticket prefix sums, table sides (build)
    tsI: object = None                 # device u64[nmod+1] ticket prefix sums, probing sides
    tsIr: object = None                # the same per radius {r: prefix sums over that radius's moduli}
    tsD_all: object = None             # table-side tickets with every modulus built in place
    tsS: object = None                 # scatter tickets of the partitioned build per radius {r: prefix sums}
    tsP: object = None                 # bucket ranges of the partitioned build (0 for in-place moduli)
    n_part: int = 0                    # moduli of this batch with the partitioned build
    use_part: bool = True              # False after a bucket range overflowed: build in place
    zero_bytes: int = 0                # arena bytes zeroed before the build
    arena_bytes: int = 0
    records: int = 0
    graph: object = None
    bset: int = 0                      # buffer set (arena, counters, pair buffers, stream) of the batch


@dataclass
class PreparedPortfolio:
    instances: list
    i_limit: int | None
    nD: list
    nI: list
    shapes: list                       # (bbits, fbits) per modulus, None when not batched
    batches: list
    fallback: list                     # portfolio positions solved one at a time (r > max or both sides >= 2^32)
    trivial: dict                      # position -> SolveResult (r = 0 or an empty side)
    tables: object = None              # device blob of pool and screen tables (kept alive)
    tails: object = None               # device blob of tail tables (kept alive)
    pairs_cap: int = 0

    @property
    def records(self) -> int:
        return sum(self.nD[k] + self.nI[k] for k in range(len(self.instances)))


class BatchSolver:
    """Solves portfolios of moduli on one device and stream with the batched kernels."""

    def __init__(self, device=None, stream=None, tuning: BatchTuning | None = None):
        import torch
        self.torch = torch
        self.lib = _lib.load()
        self.device = torch.device(device if device is not None else "cuda")
        if self.device.type != "cuda":
            raise RuntimeError("the batched join runs on a CUDA device only")
        self.stream = stream
        self.tuning = tuning or BatchTuning()
        if self.tuning.ticket <= 0 or self.tuning.ticket % 32:
            raise ValueError("ticket must be a positive multiple of 32")
        assert self.lib.cf_batch_mod_bytes() == MOD_DTYPE.itemsize
        self.max_r = self.lib.cf_batch_max_r()
        self.result_bytes = self.lib.cf_pair_result_bytes()
        self._bufs: dict = {}
        self._set = 0                  # buffer set of the batch being queued or collected
        self._set_streams: list = []
        self._capture = None           # the stream a CUDA graph is being captured on
        self._single: Solver | None = None

    # -- buffers -------------------------------------------------------------
    def _buf(self, name: str, nbytes: int):
        key = (name, self._set)
        t = self._bufs.get(key)
        if t is None or t.numel() < nbytes:
            self._drop_graphs()
            with self.torch.cuda.stream(self._torch_stream()):
                t = self.torch.empty(max(nbytes, 16), dtype=self.torch.uint8, device=self.device)
            self._bufs[key] = t
        return t

    def _nsets(self) -> int:
        return 2 if self.tuning.overlap else 1

    def _stream_of(self, k: int):
        """The stream of buffer set k: the solver's stream for one set, else one of two own streams."""
        if self._nsets() == 1:
            return self.stream if self.stream is not None else self.torch.cuda.current_stream(self.device)
        while len(self._set_streams) < 2:
            self._set_streams.append(self.torch.cuda.Stream(self.device))
        return self._set_streams[k]

    def _drop_graphs(self):
        for prep in getattr(self, "_live", []):
            for b in prep.batches:
                b.graph = None

    def _sh(self):
        return _lib.stream_handle(self._torch_stream())

    def _torch_stream(self):
        if self._capture is not None:
            return self._capture
        if self._nsets() > 1 and self._set_streams:
            return self._set_streams[self._set]
        return self.stream if self.stream is not None else self.torch.cuda.current_stream(self.device)

    def _base_stream(self):
        return self.stream if self.stream is not None else self.torch.cuda.current_stream(self.device)

    # -- preparation ---------------------------------------------------------
    def prepare(self, instances: list, i_limit: int | None = None) -> PreparedPortfolio:
        """Host tables of every modulus, one upload, device tail tables, batch split."""
        torch, lib = self.torch, self.lib
        tu = self.tuning
        insts = [w if isinstance(w, Instance) else Instance.build(w.M, w.Q, w.B0, w.r, w.B) for w in instances]
        N = len(insts)
        nD = [ncomb(len(x.B0), x.r) if x.r else 1 for x in insts]
        nI = [ncomb(len(x.INS), x.r) if x.r else 1 for x in insts]
        if i_limit is not None:
            nI = [min(v, int(i_limit)) for v in nI]
        shapes: list = [None] * N
        trivial: dict = {}
        fallback: list = []
        batched: list = []
        for k, x in enumerate(insts):
            if x.r == 0 or nD[k] == 0 or nI[k] == 0:
                trivial[k] = None
            elif x.r > self.max_r or min(nD[k], nI[k]) >= 1 << 32:
                fallback.append(k)
            else:
                shapes[k] = dtab_shape(min(nD[k], nI[k]), tu.dtab)     # the table holds the smaller side
                batched.append(k)
        # host tables packed into one blob (pools and screens), uploaded once
        host_parts, offs, off = [], {}, 0
        for k in batched:
            x = insts[k]
            multD = pow(x.P0, -1, x.M)
            for tag, arr in (("pD", pool_table_host(x.B0, x.r, x.M, multD)),
                             ("pI", pool_table_host(x.INS, x.r, x.M, 1)),
                             ("sc", screen_table_host(x.P0, x.B, 1e-6))):
                offs[(k, tag)] = off
                host_parts.append((off, arr))
                off = _up(off + arr.nbytes)
        blob_host = np.zeros(max(off, 16), dtype=np.uint8)
        for o, arr in host_parts:
            blob_host[o:o + arr.nbytes] = arr.view(np.uint8)
        blob = torch.from_numpy(blob_host).to(self.device)
        base = blob.data_ptr()
        # tail tables, built on the device from the uploaded pools
        toffs, toff = {}, 0
        for k in batched:
            x = insts[k]
            for tag, n in (("tD", len(x.B0)), ("tI", len(x.INS))):
                toffs[(k, tag)] = toff
                toff = _up(toff + lib.cf_tail_bytes(n, x.r))
        tails = torch.empty(max(toff, 16), dtype=torch.uint8, device=self.device)
        tbase = tails.data_ptr()
        sh = self._sh()
        for k in batched:
            x = insts[k]
            _lib.check(lib.cf_build_tail(base + offs[(k, "pD")], len(x.B0), x.r, tbase + toffs[(k, "tD")], sh),
                       "cf_build_tail(D)")
            _lib.check(lib.cf_build_tail(base + offs[(k, "pI")], len(x.INS), x.r, tbase + toffs[(k, "tI")], sh),
                       "cf_build_tail(I)")
        # partitioned build: (ranges, range capacity) per modulus, None when built in place
        plb = tu.part_lb
        if not lib.cf_batch_part_buckets(plb):
            raise ValueError(f"part_lb {plb} is not supported by the partitioned build")
        part: dict = {}
        for k in batched:
            bb, _fb = shapes[k]
            if tu.part_build and (1 << bb) >= tu.part_min_buckets:
                ps = part_shape(min(nD[k], nI[k]), bb, plb, tu.part_sigma, lib.cf_batch_part_max_ranges())
                if ps is not None:
                    part[k] = ps
        # batches: consecutive moduli whose D tables fit the budget
        batches, cur, cur_bytes = [], [], 0
        for k in batched:
            bb, fb = shapes[k]
            nbytes = _up(36 << bb) + (_up(32 << fb) if fb else 0) + _up(128 << bb)
            if k in part:
                npt, cap = part[k]
                nbytes += _up(npt * 4) + _up(npt * cap * 4) + _up(npt * cap * 8)
            if cur and cur_bytes + nbytes > tu.mem_budget:
                batches.append(_Batch(cur))
                cur, cur_bytes = [], 0
            cur.append(k)
            cur_bytes += nbytes
        if cur:
            batches.append(_Batch(cur))
        # descriptors with arena offsets (arena pointers are filled in at run time)
        for b in batches:
            zoff, soff_rel, poff_rel = 0, 0, 0
            rows = np.zeros(len(b.idx), dtype=MOD_DTYPE)
            zl, sl, pl = [], [], []
            for j, k in enumerate(b.idx):
                x = insts[k]
                bb, fb = shapes[k]
                zl.append(zoff)
                zoff += _up(36 << bb) + (_up(32 << fb) if fb else 0)
                if k in part:                      # range counters sit in the zeroed region
                    zoff += _up(part[k][0] * 4)
                sl.append(soff_rel)
                soff_rel += _up(128 << bb)
                pl.append(poff_rel)
                if k in part:
                    npt, cap = part[k]
                    poff_rel += _up(npt * cap * 4) + _up(npt * cap * 8)
                    rows[j]["pcap"] = cap
                    rows[j]["plb"] = plb
                rows[j]["poolD"] = base + offs[(k, "pD")]
                rows[j]["poolI"] = base + offs[(k, "pI")]
                rows[j]["screen"] = base + offs[(k, "sc")]
                rows[j]["tailD"] = tbase + toffs[(k, "tD")]
                rows[j]["tailI"] = tbase + toffs[(k, "tI")]
                rows[j]["nD"] = nD[k]
                rows[j]["i_lo"] = 0
                rows[j]["nI"] = nI[k]
                rows[j]["bbits"], rows[j]["fbits"], rows[j]["r"] = bb, fb, x.r
                rows[j]["swap"] = int(nI[k] < nD[k])
            b.zero_bytes = zoff
            b.arena_bytes = zoff + soff_rel + poff_rel
            b.records = sum(nD[k] + nI[k] for k in b.idx)
            b._rows, b._zl, b._sl, b._pl = rows, zl, sl, pl
            b._side_bytes = soff_rel
            b._part = {j: part[k] for j, k in enumerate(b.idx) if k in part}
            b.n_part = len(b._part)
            t = tu.ticket
            tile = lib.cf_batch_part_tile()

            def _prefix(vals):
                a = np.zeros(len(b.idx) + 1, dtype=np.uint64)
                a[1:] = np.cumsum(vals)
                return torch.from_numpy(a.view(np.int64)).to(self.device)
            # mode 0 walks the table's (smaller) side, mode 1 the probing side; the
            # partitioned build takes the table sides of the moduli in b._part
            build = [-(-min(nD[k], nI[k]) // t) for k in b.idx]
            b.tsD_all = _prefix(build)
            b.tsD = _prefix([0 if j in b._part else v for j, v in enumerate(build)])
            b.tsI = _prefix([-(-max(nD[k], nI[k]) // t) for k in b.idx])
            # the probe runs one launch per radius present, each over its radius's moduli only
            b.tsIr = {rr: _prefix([-(-max(nD[k], nI[k]) // t) if insts[k].r == rr else 0 for k in b.idx])
                      for rr in sorted({insts[k].r for k in b.idx})}
            # one scatter launch per radius present, each with a generator specialised for it
            b.tsS = {}
            for rr in sorted({insts[k].r for j, k in enumerate(b.idx) if j in b._part}):
                b.tsS[rr] = _prefix([-(-min(nD[k], nI[k]) // tile) if j in b._part and insts[k].r == rr else 0
                                     for j, k in enumerate(b.idx)])
            b.tsP = _prefix([b._part[j][0] if j in b._part else 0 for j in range(len(b.idx))])
        prep = PreparedPortfolio(insts, i_limit, nD, nI, shapes, batches, fallback, trivial, blob, tails,
                                 tu.pair_capacity)
        self._place(prep)
        self._live = getattr(self, "_live", []) + [prep]
        return prep

    def _place(self, prep: PreparedPortfolio):
        """Point every batch's descriptors into the arena of its buffer set and upload them
        (with overlap, consecutive batches alternate between two sets)."""
        torch = self.torch
        if not prep.batches:
            return
        nsets = self._nsets()
        saved = self._set
        try:
            for k in range(nsets):
                mine = [bt for i, bt in enumerate(prep.batches) if i % nsets == k]
                if not mine:
                    continue
                self._set = k
                arena = self._buf("arena", max(bt.arena_bytes for bt in mine))
                abase = arena.data_ptr()
                for bt in mine:
                    bt.bset = k
                    rows = bt._rows.copy()
                    for j, kk in enumerate(bt.idx):
                        bb, fb = prep.shapes[kk]
                        z = abase + bt._zl[j]
                        rows[j]["fpw"] = z
                        rows[j]["fill"] = z + (32 << bb)
                        rows[j]["bloom"] = z + _up(36 << bb) if fb else 0
                        rows[j]["side"] = abase + bt.zero_bytes + bt._sl[j]
                        if j in bt._part:
                            npt, cap = bt._part[j]
                            rows[j]["pcnt"] = z + _up(36 << bb) + (_up(32 << fb) if fb else 0)
                            pk = abase + bt.zero_bytes + bt._side_bytes + bt._pl[j]
                            rows[j]["pkw"] = pk
                            rows[j]["psd"] = pk + _up(npt * cap * 4)
                    bt.mods = torch.from_numpy(rows.view(np.uint8).copy()).to(self.device)
                    bt._arena_ptr = abase
        finally:
            self._set = saved

    # -- running -------------------------------------------------------------
    def _enqueue(self, b: _Batch, maxp: int):
        """Queue the batch's whole device sequence with one cf_solve_batch call."""
        import ctypes as C
        lib, dp = self.lib, _lib.ptr
        arena = self._bufs[("arena", self._set)]
        misc = self._buf("misc", 64)
        ovf = self._buf("ovf", tu_ovf_bytes(self))
        pairs = self._buf("pairs", maxp * 16)
        pmod = self._buf("pmod", maxp * 4)
        res = self._buf("res", maxp * self.result_bytes)
        tu = self.tuning
        part = b.use_part and b.n_part > 0
        scat = sorted(b.tsS.items()) if part else []
        s_ptrs = (C.c_void_p * max(1, len(scat)))(*[dp(ts) for _, ts in scat])
        s_rad = (C.c_int * max(1, len(scat)))(*[int(rr) for rr, _ in scat])
        prb = sorted(b.tsIr.items()) if (tu.probe_per_radius and b.tsIr) else []
        p_ptrs = (C.c_void_p * max(1, len(prb)))(*[dp(ts) for _, ts in prb])
        p_rad = (C.c_int * max(1, len(prb)))(*[int(rr) for rr, _ in prb])
        q = _lib.CfBatchQueue(
            mods=dp(b.mods), arena=dp(arena), zero_bytes=b.zero_bytes, misc=dp(misc),
            build_tickets=dp(b.tsD if part else b.tsD_all), probe_tickets=dp(b.tsI),
            place_tickets=dp(b.tsP) if part else None, scatter_tickets=C.addressof(s_ptrs),
            scatter_radius=C.addressof(s_rad), ovf=dp(ovf), pairs=dp(pairs), pair_mods=dp(pmod), results=dp(res),
            nmod=len(b.idx), ticket=tu.ticket, grid=tu.grid, max_pairs=maxp, ovf_cap=tu.ovf_capacity,
            n_scatter=len(scat), use_part=int(part), part_lb=tu.part_lb, n_probe=len(prb),
            probe_tickets_r=C.addressof(p_ptrs), probe_radius=C.addressof(p_rad))
        _lib.check(lib.cf_solve_batch(C.byref(q), self._sh()), "cf_solve_batch")

    def _launch(self, b: _Batch, maxp: int, graphs: bool):
        """Queue batch b on the stream of its buffer set (replaying its CUDA graph when graphs)."""
        torch = self.torch
        self._set = b.bset
        if not graphs:
            self._enqueue(b, maxp)
            return
        if b.graph is None or b._graph_maxp != maxp or b._arena_ptr != self._bufs[("arena", b.bset)].data_ptr():
            for nm, nb in (("misc", 64), ("ovf", tu_ovf_bytes(self)), ("pairs", maxp * 16), ("pmod", maxp * 4),
                           ("res", maxp * self.result_bytes)):
                self._buf(nm, nb)            # allocate outside the capture
            g = torch.cuda.CUDAGraph()
            home = self._torch_stream()
            s = torch.cuda.Stream(self.device)
            s.wait_stream(home)
            with torch.cuda.stream(s):
                self._capture = s
                try:
                    with torch.cuda.graph(g, stream=s):
                        self._enqueue(b, maxp)
                finally:
                    self._capture = None
            home.wait_stream(s)
            b.graph, b._graph_maxp = g, maxp
        with torch.cuda.stream(self._torch_stream()):
            b.graph.replay()

    def _drain(self):
        for k in range(self._nsets()):
            self._stream_of(k).synchronize()

    def run(self, prep: PreparedPortfolio, verify: bool = True, graphs: bool = False,
            marks: list | None = None) -> list[SolveResult]:
        """Every result of the portfolio, in input order.  With overlap, batch i + 1 is queued on
        the other buffer set and stream before batch i is collected: its table builds run beside
        batch i's probes, and the host's certification of batch i beside its kernels."""
        torch = self.torch
        out: list = [None] * len(prep.instances)
        for k in prep.trivial:
            out[k] = self._trivial(prep, k, verify)
        base = self._base_stream()
        for k in range(self._nsets()):
            st = self._stream_of(k)
            if st is not base:
                st.wait_stream(base)            # after the preparation's uploads and tail builds
        saved = self._set
        pending = None
        try:
            for b in prep.batches:
                if pending is not None and pending.bset == b.bset:
                    self._collect(prep, pending, graphs, verify, out, marks)   # b reuses its buffers
                    pending = None
                if b._arena_ptr != self._bufs[("arena", b.bset)].data_ptr():
                    self._drain()               # another portfolio moved the arenas: place this one again
                    self._place(prep)
                self._launch(b, prep.pairs_cap, graphs)
                if marks is not None:
                    ev = torch.cuda.Event(enable_timing=True)
                    ev.record(self._torch_stream())
                    marks.append(("batch", ev))
                if pending is not None:
                    self._collect(prep, pending, graphs, verify, out, marks)
                pending = b
            if pending is not None:
                self._collect(prep, pending, graphs, verify, out, marks)
        finally:
            self._set = saved
            for k in range(self._nsets()):
                st = self._stream_of(k)
                if st is not base:
                    base.wait_stream(st)        # work queued after run() follows every batch
        if prep.fallback:
            if self._single is None:
                self._single = Solver(self.device, self.stream, self.tuning.dtab)
            for k in prep.fallback:
                out[k] = self._single.solve_instance(prep.instances[k], verify=verify, i_limit=prep.i_limit)
        return out

    def _collect(self, prep: PreparedPortfolio, b: _Batch, graphs: bool, verify: bool, out: list, marks):
        """Read batch b's counters on its own stream (the other batch keeps running), re-run it on
        an overflow (after draining both streams: buffers may grow), and finish its moduli."""
        torch = self.torch
        for _attempt in range(8):
            self._set = b.bset
            with torch.cuda.stream(self._torch_stream()):
                misc = self._bufs[("misc", b.bset)][:32].cpu().numpy().view(np.uint32)
            npairs, err = int(misc[4]), int(misc[5])
            retry = False
            if err & _lib.ERR_PART_OVERFLOW and b.use_part and b.n_part:
                b.use_part, b.graph = False, None       # a bucket range overflowed: build in place
                retry = True
            elif err & _lib.ERR_PAIR_OVERFLOW:
                prep.pairs_cap = 1 << max(npairs + 16, 2 * prep.pairs_cap).bit_length()
                retry = True
            elif err & _lib.ERR_TABLE_FULL:
                raise _lib.CfError(_lib.CF_EOVERFLOW, "batch", "D table full (internal error)")
            elif err:
                raise _lib.CfError(_lib.CF_EBADARG, "batch", f"a batched kernel rejected its work (err {err:#x})")
            if not retry:
                break
            if _attempt == 7:
                raise _lib.CfError(_lib.CF_EOVERFLOW, "batch", "pair buffer kept overflowing")
            self._drain()
            self._launch(b, prep.pairs_cap, graphs)
            if marks is not None:
                ev = torch.cuda.Event(enable_timing=True)
                ev.record(self._torch_stream())
                marks.append(("batch", ev))
        self._set = b.bset
        with torch.cuda.stream(self._torch_stream()):
            rows = np.frombuffer(self._bufs[("res", b.bset)][: npairs * self.result_bytes].cpu().numpy().tobytes(),
                                 dtype=RESULT_DTYPE)
            mods = self._bufs[("pmod", b.bset)][: npairs * 4].cpu().numpy().view(np.uint32)
        order = np.argsort(mods, kind="stable")
        rows, mods = rows[order], mods[order]
        cuts = np.searchsorted(mods, np.arange(len(b.idx) + 1))
        for j, k in enumerate(b.idx):
            bb, fb = prep.shapes[k]
            plan = dict(strategy="fused", batched=True, bbits=bb, fbits=fb, i_limit=prep.i_limit)
            out[k] = finish_rows(prep.instances[k], rows[cuts[j]:cuts[j + 1]], prep.nD[k], prep.nI[k], plan,
                                 verify)

    def _trivial(self, prep: PreparedPortfolio, k: int, verify: bool) -> SolveResult:
        x = prep.instances[k]
        if x.r == 0:
            if self._single is None:
                self._single = Solver(self.device, self.stream, self.tuning.dtab)
            return self._single._solve_r0(x)
        return SolveResult([], prep.nD[k], prep.nI[k], 0, 0, 0, 0)

    def solve(self, instances: list, i_limit: int | None = None, verify: bool = True,
              graphs: bool = False) -> list[SolveResult]:
        return self.run(self.prepare(instances, i_limit), verify=verify, graphs=graphs)

    def release(self, prep: PreparedPortfolio):
        """Drop a prepared portfolio's graphs and device tables."""
        for b in prep.batches:
            b.graph = None
            b.mods = b.tsD = b.tsI = b.tsD_all = b.tsS = b.tsP = b.tsIr = None
        prep.tables = prep.tails = None
        live = getattr(self, "_live", [])
        self._live = [p for p in live if p is not prep]


# -- per-modulus forms, for comparison ------------------------------------------

def run_per_modulus(instances: list, i_limit: int | None = None, verify: bool = True, device=None,
                    solver: Solver | None = None) -> list[SolveResult]:
    """This library's single-modulus fused solve, one modulus at a time on the device (the host
    collects each solve while the next one runs: Solver.solve_many)."""
    s = solver or Solver(device)
    xs = [w if isinstance(w, Instance) else Instance.build(w.M, w.Q, w.B0, w.r, w.B) for w in instances]
    return s.solve_many(xs, verify=verify, i_limit=i_limit)


def run_plain(instances: list, i_limit: int | None = None, verify: bool = True, chunk: int = 1 << 27,
              device=None) -> list[SolveResult]:
    """The reference's per-modulus GPU form: generate -> sort_side -> join_sorted on each side
    (gpu/mitm_gpu2.py:79-119 as driven by gpu/mitm_gpu_mstar_driver.py:184-286), keys
    prod(D) and P0 * prod(I) mod M, exact check of every pair on the host."""
    from . import mitm_gpu2 as G
    out = []
    for w in instances:
        x = w if isinstance(w, Instance) else Instance.build(w.M, w.Q, w.B0, w.r, w.B)
        r, M = x.r, x.M
        nD = ncomb(len(x.B0), r)
        nI = ncomb(len(x.INS), r)
        if i_limit is not None:
            nI = min(nI, int(i_limit))
        if r == 0 or nD == 0 or nI == 0:
            out.append(SolveResult([], nD, nI, 0, 0, 0, 0))
            continue
        bits = max(6, (max(len(x.B0), len(x.INS)) - 1).bit_length())
        Dk, Did = G.sort_side(*G.generate(x.B0, r, M, 1, bits, device=device))
        pairs = []
        for lo in range(0, nI, chunk):
            hi = min(nI, lo + chunk)
            Ik, Iid = G.sort_side(*G.generate(x.INS, r, M, x.P0 % M, bits, lo, hi, device=device))
            d_ids, i_ids = G.join_sorted(Dk, Did, Ik, Iid)
            if d_ids.numel():
                pairs += list(zip(G.decode_ids(d_ids, r, bits), G.decode_ids(i_ids, r, bits)))
            del Ik, Iid
        hits, above, rejected, plist = [], 0, 0, []
        for di, ii in pairs:
            D = tuple(x.B0[i] for i in di)
            I = tuple(x.INS[i] for i in ii)
            plist.append((D, I))
            dset = set(D)
            fac = tuple(sorted([p for p in x.B0 if p not in dset] + list(I)))
            n = math.prod(fac)
            if n > x.B:
                above += 1
                continue
            ok = (n - 1) % M == 0
            if ok and verify:
                ok, n2, _ = verify_certificate(fac)
                ok = ok and n2 == n
            if ok:
                hits.append(Hit(D, I, n, fac))
            else:
                rejected += 1
        hits.sort(key=lambda h: (h.n, h.D, h.I))
        plist.sort()
        out.append(SolveResult(hits, nD, nI, len(plist), len(plist) - above, above, rejected,
                               plan=dict(strategy="plain"), pairs=plist))
    return out
