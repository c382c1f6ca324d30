"""Serving loop: continuous batching of modulus-solve requests on one GPU.

Requests (M, Q, B0, r, B) arrive over time.  The loop admits a request when a
worker slot is free and its estimated HBM footprint fits in the memory budget;
admitted requests run concurrently, each on its own CUDA stream and worker
thread, so the device works on several of them at once and a new request starts
as soon as a slot and memory free up -- not when a batch ends.  Pool tables stay
resident on the device in each worker's table cache.

Footprint estimates are upper bounds computed on the host before any device
work: the bounded solve's side sizes are bounded by a dynamic programme over
rounded log2 prime sizes (counts of r-subsets whose rounded log-product passes
the bound, rounded so that the count can only be too large), and the fused
solve's table by C(n, r).  A request whose estimate exceeds the whole budget
runs alone.

The reference has no serving loop: its drivers solve one instance after another
(gpu/mitm_gpu_mstar_driver.py:296-320).  ``run_serial`` is that form, and
``run_poisson`` drives either form with Poisson arrivals and reports p50/p99
latency and throughput.
"""
from __future__ import annotations

import math
import random
import threading
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from .solve import Instance, SolveResult, Tuning

LOG_STEP = 0.25          # bits per weight unit of the size-bound dynamic programme


# -- footprint estimate --------------------------------------------------------------

def _count_dp(weights, r: int, cap: int, at_least: bool) -> int:
    """Number of r-subsets whose weight sum is >= cap (at_least) or <= cap (else),
    for non-negative integer weights, sums clipped at cap + 1."""
    top = cap + 1
    dp = np.zeros((r + 1, top + 1), dtype=np.float64)     # counts as floats: only an upper bound is needed
    dp[0, 0] = 1
    for u in weights:
        u = int(u)
        for c in range(r, 0, -1):
            prev = dp[c - 1]
            if at_least:
                if u >= top:
                    dp[c, top] += prev.sum()
                else:
                    dp[c, u:top] += prev[: top - u]
                    dp[c, top] += prev[top - u:].sum()
            else:
                if u <= top:
                    dp[c, u:] += prev[: top + 1 - u]
    v = float(dp[r, cap:].sum()) if at_least else float(dp[r, : cap + 1].sum())
    return int(math.ceil(v * (1 + 1e-9))) + 1


def count_ge_upper(primes, r: int, lower: int) -> int:
    """Upper bound on the r-subsets with product >= lower (log2 sizes rounded up)."""
    if lower <= 1:
        return math.comb(len(primes), r)
    w = [math.ceil(math.log2(p) / LOG_STEP) for p in primes]
    cap = max(0, math.floor((lower.bit_length() - 1) / LOG_STEP))
    return min(math.comb(len(primes), r), _count_dp(w, r, cap, True))


def count_lt_upper(primes, r: int, cap_excl: int) -> int:
    """Upper bound on the r-subsets with product < cap_excl (log2 sizes rounded down)."""
    if cap_excl <= 1:
        return 0
    w = [math.floor(math.log2(p) / LOG_STEP) for p in primes]
    cap = math.ceil(cap_excl.bit_length() / LOG_STEP)
    return min(math.comb(len(primes), r), _count_dp(w, r, cap, False))


def _dtab_bytes(n: int, tu: Tuning) -> int:
    from .solve import dtab_shape
    bb, fb = dtab_shape(max(n, 1), tu)
    return (164 << bb) + ((32 << fb) if fb else 0)


def footprint(inst: Instance, tu: Tuning) -> dict:
    """Upper bound on the device bytes one solve of `inst` holds at once, and the
    strategy it will use ('bounded' or 'fused')."""
    from . import bsolve
    max_nodes = tu.max_nodes
    r = inst.r
    nB, nI_full = len(inst.B0), len(inst.INS)
    fixed = 64 << 20                                          # pools, tails, pair buffers, scan space
    if r == 0:
        return dict(bytes=fixed, strategy="host")
    if tu.strategy in ("auto", "bounded") and bsolve.applicable(inst) and \
            (tu.strategy == "bounded" or bsolve.prunes(inst)):
        Icap, Dmin = bsolve.caps(inst)
        nD = count_ge_upper(inst.B0, r, Dmin)
        nI = count_lt_upper(inst.INS, r, Icap)
        frontier = 40 * min(max_nodes, max(nD, nI))           # one frontier block of nodes
        # table on the I leaves (written only when they are fewer than the D records, so at
        # most min(nI, nD) of them) or on the D records (I leaves probed, never written)
        m = min(nI, nD)
        side = max(16 * m + _dtab_bytes(m, tu), _dtab_bytes(nD, tu))
        return dict(bytes=fixed + 16 * nD + frontier * 2 + side, strategy="bounded", nD=nD, nI=nI, work=nD + nI)
    small = min(math.comb(nB, r), math.comb(nI_full, r))
    tails = 16 * (math.comb(nB, 2) + math.comb(nI_full, 2))
    return dict(bytes=fixed + _dtab_bytes(small, tu) + tails, strategy="fused",
                work=math.comb(nB, r) + math.comb(nI_full, r))


# -- admission and workers ---------------------------------------------------------

@dataclass
class Ticket:
    rid: int
    inst: Instance
    arrival: float
    need: int = 0
    work: int = 0                       # estimated records (footprint()["work"])
    admitted: float = 0.0
    finished: float = 0.0
    result: SolveResult | None = None
    error: str | None = None
    exclusive: bool = False
    large: bool = False                 # runs in the large lane (one at a time, high priority)
    done: threading.Event = field(default_factory=threading.Event)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class Admission:
    """Byte budget and FIFO queue with bounded bypass: a worker takes the oldest
    waiting request whose footprint fits; a request that has been passed over
    `max_bypass` times blocks younger ones until it fits.  A request larger than
    the budget runs alone.  Large requests (Ticket.large) run one at a time in
    arrival order -- the tail of the latency distribution is theirs, and two of
    them sharing the GPU both finish late -- while younger small ones pass a large
    request that waits for the lane; while a large request runs, at most
    `beside_large` small ones (None: any number) run beside it."""

    def __init__(self, budget: int, max_bypass: int = 8, beside_large: int | None = None):
        self.budget = int(budget)
        self.used = 0
        self.running = 0
        self.large_running = 0
        self.beside_large = beside_large      # small requests admitted while a large one runs (None: any)
        self.peak = 0
        self.max_bypass = max_bypass
        self.q: deque = deque()
        self.bypassed: dict = {}
        self.cv = threading.Condition()
        self.closed = False

    def put(self, t: Ticket):
        with self.cv:
            t.exclusive = t.need > self.budget
            self.q.append(t)
            self.cv.notify_all()

    def close(self):
        with self.cv:
            self.closed = True
            self.cv.notify_all()

    def _pick(self):
        for i, t in enumerate(self.q):
            if t.large and not t.exclusive and self.large_running:
                continue             # the large lane is busy: younger requests may pass, not counted as bypass
            if (not t.large and self.large_running and self.beside_large is not None
                    and self.running - self.large_running >= self.beside_large):
                return None          # a large request runs: only beside_large small ones share the GPU with it
            if t.exclusive:
                ok = self.running == 0
            else:
                ok = self.used + t.need <= self.budget
            if ok:
                for older in list(self.q)[:i]:
                    self.bypassed[older.rid] = self.bypassed.get(older.rid, 0) + 1
                del self.q[i]
                return t
            if self.bypassed.get(t.rid, 0) >= self.max_bypass or t.exclusive:
                return None          # this one waits at the head; nobody passes it any more
        return None

    def take(self) -> Ticket | None:
        with self.cv:
            while True:
                t = self._pick()
                if t is not None:
                    # a request larger than the budget takes all of it: nothing runs beside it
                    self.used += self.budget if t.exclusive else t.need
                    self.running += 1
                    self.large_running += int(t.large)
                    self.peak = max(self.peak, self.used)
                    self.bypassed.pop(t.rid, None)
                    return t
                if self.closed and not self.q:
                    return None
                self.cv.wait(0.05)

    def release(self, t: Ticket):
        with self.cv:
            self.used -= self.budget if t.exclusive else t.need
            self.running -= 1
            self.large_running -= int(t.large)
            self.cv.notify_all()


class Server:
    """Continuous-batching solve server on one device.

    slots: concurrent requests (one worker thread and CUDA stream each);
    budget: device bytes that admitted requests may hold together (default: 60%
    of the free device memory at start); solve_fn(worker_state, inst) may replace
    the GPU solve (used by CPU tests of the admission logic).
    large_work: requests whose estimated records (footprint()["work"]) reach this are large: they
    run one at a time (Admission), so that the largest requests -- the tail of the latency
    distribution -- do not share the GPU with one another, while the small ones fill the SMs a
    large one leaves free; beside_large caps the small requests that run while a large one does
    (None: any); priority: which requests take the worker's high-priority stream ("large",
    "small" or "none"; measured on the seeded stream at 3 req/s, "none" and "small" give the
    small requests a p50 of 14 ms against 37 ms when the large ones take it, at the same p99).
    The default large_work is the measured knee of the seeded serving stream: its requests above
    3e9 estimated records take 0.2-1.7 s alone and are about a sixth of the stream, those below
    take milliseconds."""

    def __init__(self, device=None, slots: int = 4, budget: int | None = None, strategy: str = "auto",
                 solve_fn=None, clock=time.perf_counter, large_work: float = 3e9,
                 beside_large: int | None = None, priority: str = "none"):
        if priority not in ("large", "small", "none"):
            raise ValueError("priority must be 'large', 'small' or 'none'")
        self.slots = slots
        self.large_work = large_work
        self.priority = priority
        self.clock = clock
        self.tuning = Tuning(strategy=strategy, max_nodes=1 << 22)
        self.solve_fn = solve_fn
        self.device = device
        if budget is None:
            import torch
            free, _total = torch.cuda.mem_get_info(torch.device(device if device is not None else "cuda"))
            budget = int(free * 0.6)
        self.adm = Admission(budget, beside_large=beside_large)
        self.tickets: list[Ticket] = []
        self._rid = 0
        self._threads: list[threading.Thread] = []
        self._lock = threading.Lock()

    # -- lifecycle -------------------------------------------------------------
    def start(self):
        for w in range(self.slots):
            th = threading.Thread(target=self._worker, args=(w,), daemon=True)
            th.start()
            self._threads.append(th)
        return self

    def stop(self):
        self.adm.close()
        for th in self._threads:
            th.join()
        self._threads = []

    def submit(self, inst: Instance, arrival: float | None = None) -> Ticket:
        with self._lock:
            rid = self._rid
            self._rid += 1
        t = Ticket(rid, inst, self.clock() if arrival is None else arrival)
        if self.solve_fn is None:
            fp = footprint(inst, self.tuning)
            t.need, t.work = fp["bytes"], fp.get("work", 0)
        else:
            t.need, t.work = getattr(inst, "need", 1), getattr(inst, "work", 0)
        t.large = t.work >= self.large_work
        self.tickets.append(t)
        self.adm.put(t)
        return t

    # -- workers ---------------------------------------------------------------
    def _worker(self, w: int):
        state = self._worker_state(w)
        while True:
            t = self.adm.take()
            if t is None:
                return
            t.admitted = self.clock()
            try:
                fast = (self.priority == "large" and t.large) or (self.priority == "small" and not t.large)
                t.result = self._solve(state, t.inst, fast)
            except Exception as e:                     # noqa: BLE001 - reported per request
                t.error = f"{type(e).__name__}: {e}"
            finally:
                self._trim(state)
                t.finished = self.clock()
                self.adm.release(t)
                t.done.set()

    def _worker_state(self, w: int):
        if self.solve_fn is not None:
            return {"worker": w}
        import torch
        from .solve import Solver
        dev = torch.device(self.device if self.device is not None else "cuda")
        lo, hi = torch.cuda.Stream.priority_range()
        stream = torch.cuda.Stream(dev)
        fast = torch.cuda.Stream(dev, priority=hi)           # the highest priority the device offers
        return {"worker": w, "stream": stream, "solver": Solver(dev, stream=stream, tuning=self.tuning),
                "fast_stream": fast, "fast_solver": Solver(dev, stream=fast, tuning=self.tuning)}

    def _solve(self, state, inst: Instance, fast: bool = False) -> SolveResult:
        """Solve on the worker's high-priority stream (fast) or its normal one."""
        if self.solve_fn is not None:
            return self.solve_fn(state, inst)
        import torch
        st, solver = (state["fast_stream"], state["fast_solver"]) if fast else (state["stream"], state["solver"])
        with torch.cuda.stream(st):
            res = solver.solve_instance(inst)
            st.synchronize()
        return res

    def _trim(self, state):
        """Drop the worker's per-request device buffers (pool tables stay resident)."""
        for key in ("solver", "fast_solver"):
            s = state.get(key)
            if s is not None:
                s._bufs.clear()


# -- drivers ------------------------------------------------------------------------

def poisson_arrivals(n: int, rate: float, seed: int = 0) -> list[float]:
    rng = random.Random(seed)
    t, out = 0.0, []
    for _ in range(n):
        t += rng.expovariate(rate)
        out.append(t)
    return out


def _stats(tickets: list, t0: float, t_end: float) -> dict:
    lat = sorted(1e3 * t.latency for t in tickets)
    n = len(lat)
    pick = lambda q: lat[min(n - 1, int(math.ceil(q * n)) - 1)] if n else None   # noqa: E731
    return dict(requests=n, p50_ms=pick(0.50), p99_ms=pick(0.99), mean_ms=sum(lat) / n if n else None,
                throughput_rps=n / (t_end - t0) if t_end > t0 else None,
                errors=sum(1 for t in tickets if t.error),
                hits=sum(len(t.result.hits) for t in tickets if t.result is not None))


def run_poisson(server: Server, insts: list, rate: float, seed: int = 0) -> dict:
    """Submit `insts` at Poisson arrival times (rate per second) and wait for all."""
    arr = poisson_arrivals(len(insts), rate, seed)
    t0 = server.clock()
    tickets = []
    for inst, a in zip(insts, arr):
        now = server.clock() - t0
        if a > now:
            time.sleep(a - now)
        tickets.append(server.submit(inst, arrival=t0 + a))
    for t in tickets:
        t.done.wait()
    t_end = max(t.finished for t in tickets) if tickets else t0
    out = _stats(tickets, t0, t_end)
    out.update(offered_rps=rate, slots=server.slots, peak_reserved=server.adm.peak, budget=server.adm.budget)
    return out, tickets


def run_serial(solve, insts: list, rate: float, seed: int = 0, clock=time.perf_counter) -> tuple[dict, list]:
    """The serial form: one request at a time, in arrival order, with the same
    Poisson arrivals (a request waits while an earlier one runs)."""
    arr = poisson_arrivals(len(insts), rate, seed)
    t0 = clock()
    tickets = []
    for rid, (inst, a) in enumerate(zip(insts, arr)):
        now = clock() - t0
        if a > now:
            time.sleep(a - now)
        t = Ticket(rid, inst, t0 + a)
        t.admitted = clock()
        try:
            t.result = solve(inst)
        except Exception as e:                         # noqa: BLE001
            t.error = f"{type(e).__name__}: {e}"
        t.finished = clock()
        tickets.append(t)
    t_end = max(t.finished for t in tickets) if tickets else t0
    out = _stats(tickets, t0, t_end)
    out.update(offered_rps=rate, slots=1)
    return out, tickets


def plain_solve(inst: Instance, device=None, chunk: int = 1 << 27) -> SolveResult:
    """The reference's per-instance GPU form on the filtered sides, one request at a
    time: Dmin-filtered D records, sort_side; Icap-filtered I records in chunks
    (igen_gpu.generate_chunks), sort_side, join_sorted against D; exact host check
    of every pair (gpu/mitm_gpu_mstar_driver.py:184-262, through this package's
    drop-ins for gpu/mitm_gpu2.py and gpu/igen_gpu.py)."""
    from . import bsolve, igen_gpu, mitm_gpu2 as G
    from .bounded import generator
    from .certify import verify_certificate
    from .solve import Hit
    from .tables import unrank_colex
    r, M = inst.r, inst.M
    Icap, Dmin = bsolve.caps(inst)
    Dk, Did, nD = generator(device).generate_D(inst.B0, r, M, Dmin, bitmask=2)
    Dk, Did = G.sort_side(Dk, Did)
    nI, pairs, hits, above = 0, [], [], 0
    gen = igen_gpu.generate_chunks(inst.INS, r, M, inst.P0, Icap, max_records=chunk, device=device)
    for Ik, Iid in gen:
        nI += int(Ik.numel())
        if nD == 0:
            continue
        Ik, Iid = G.sort_side(Ik, Iid)
        pd, pi = G.join_sorted(Dk, Did, Ik, Iid)
        for d, i in zip(pd.cpu().numpy().tolist() if pd.numel() else [], pi.cpu().numpy().tolist() if pi.numel() else []):
            D = tuple(inst.B0[x] for x in unrank_colex(d, r, len(inst.B0)))
            I = tuple(inst.INS[x] for x in unrank_colex(i, r, len(inst.INS)))
            pairs.append((D, I))
            dset = set(D)
            fac = tuple(sorted([p for p in inst.B0 if p not in dset] + list(I)))
            n = math.prod(fac)
            if n > inst.B:
                above += 1
                continue
            ok, n2, _ = verify_certificate(fac)
            if ok and n2 == n:
                hits.append(Hit(D, I, n, fac))
    hits.sort(key=lambda h: (h.n, h.D, h.I))
    pairs.sort()
    return SolveResult(hits, nD, nI, len(pairs), len(pairs) - above, above, 0, plan=dict(strategy="plain"),
                       pairs=pairs)

