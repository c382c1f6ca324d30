"""Census producers: which moduli a 64-factor search must run, and their batched portfolios.

The exchange join searches one family lambda(n) | M at a time; the census decides which moduli those
are.  For an incumbent U (a Carmichael number with 64 prime factors) and M = lambda(U), every
Carmichael n with 64 factors, n < U and lambda(n) | M has lambda(n) = D for some divisor D of M, all
its primes in Q(D) = {q prime : (q-1) | D, q does not divide D} and n = 1 (mod D).  A divisor can carry
such an n only if the 64 smallest primes of Q(D) multiply to less than U (a "survivor"); for a
survivor every qualifying 64-subset uses primes q <= cap(D) = (U-1) // T63(D) only (T63 = product of
the 63 smallest) and differs from the 64 smallest in at most rmax(D) places.  This restates the
reference's divisor-family census (gpu/divisor_family_census.py:45-78: the survivor test, cap, rmax
and the count s of the incumbent's primes that D forces out).  ``family_run`` then runs the rows as
gpu/run_mstar_family.py:66-94 does (the 64 smallest primes at r = 0, then radii 1..rmax over the
capped pool, bound n < U, through the driver drop-in's bounded GPU join), and ``family_instances``
hands them to the batched portfolio or the serving loop as instances.

The pools are built for all divisors at once: the candidate primes are q = d + 1 for the divisors d of
M (so (q-1) | M), each candidate's divisor exponent vector is compared with every divisor's, and q
divides D only when q is a prime of M present in D.  The reference factors and enumerates divisors of
each D separately; the rows are the same (pinned against the reference's own census output).

CPU work by nature (integer set arithmetic and 500-digit products, a few seconds per incumbent): it
supplies the moduli; the joins run on the GPU.
"""
from __future__ import annotations

import itertools
import math

import numpy as np

SIEVE_BOUND = 2_000_000          # pool primes are taken below this; a row whose cap reaches it is rejected


def _sieve(n: int) -> np.ndarray:
    s = np.ones(n + 1, dtype=bool)
    s[:2] = False
    for i in range(2, math.isqrt(n) + 1):
        if s[i]:
            s[i * i::i] = False
    return s


_SIEVE: dict = {}


def _is_prime_table(bound: int) -> np.ndarray:
    t = _SIEVE.get(bound)
    if t is None:
        t = _SIEVE[bound] = _sieve(bound)
    return t


def factorize(m: int) -> dict[int, int]:
    """Prime factorisation of m by trial division (the moduli here are products of small primes)."""
    if m < 1:
        raise ValueError("m must be positive")
    f: dict[int, int] = {}
    d = 2
    while d * d <= m:
        while m % d == 0:
            f[d] = f.get(d, 0) + 1
            m //= d
        d += 1 if d == 2 else 2
    if m > 1:
        f[m] = f.get(m, 0) + 1
    return f


def carmichael_lambda(primes) -> int:
    """lambda(n) of a squarefree n given by its primes: lcm of (p - 1)."""
    return math.lcm(*[int(p) - 1 for p in primes])


class DivisorLattice:
    """Divisors of M as exponent vectors, and the eligible pool Q(D) of every divisor D."""

    def __init__(self, M: int, sieve_bound: int = SIEVE_BOUND):
        self.M = int(M)
        self.fm = factorize(self.M)
        self.primes = sorted(self.fm)
        ranges = [range(self.fm[p] + 1) for p in self.primes]
        vecs = list(itertools.product(*ranges))
        self.E = np.asarray(vecs, dtype=np.int16).reshape(len(vecs), len(self.primes))
        values = [1]                      # same order as the exponent vectors (last prime fastest)
        for p in self.primes:
            pw = [p ** k for k in range(self.fm[p] + 1)]
            values = [v * w for v in values for w in pw]
        self.values = values
        self.index = {v: j for j, v in enumerate(values)}
        isp = _is_prime_table(sieve_bound)
        cand = [j for j, d in enumerate(self.values) if 3 <= d + 1 <= sieve_bound and isp[d + 1]]
        self.cq = np.asarray([self.values[j] + 1 for j in cand], dtype=np.int64)     # candidate primes
        self.cE = self.E[cand]                                                        # exponents of q - 1
        # q divides D only for q a prime factor of M whose exponent in D is at least 1
        self.cidx = np.asarray([self.primes.index(int(q)) if int(q) in self.fm else -1 for q in self.cq],
                               dtype=np.int64)
        order = np.argsort(self.cq)
        self.cq, self.cE, self.cidx = self.cq[order], self.cE[order], self.cidx[order]

    def pool(self, j: int) -> list[int]:
        """Q(D) below the sieve bound, ascending, for the divisor with index j."""
        e = self.E[j]
        ok = (self.cE <= e).all(axis=1)
        inM = self.cidx >= 0
        divides = np.zeros(len(self.cq), dtype=bool)
        divides[inM] = e[self.cidx[inM]] >= 1
        return [int(q) for q in self.cq[ok & ~divides]]


class SieveBoundError(ValueError):
    """A modulus whose census needs primes beyond the sieve bound."""


def census_row(D: int, P: list[int], U: int, U_factors, k: int = 64, sieve_bound: int = SIEVE_BOUND):
    """The census row of divisor D with pool P (ascending), or None when D cannot carry a k-factor
    Carmichael number below U.  Raises SieveBoundError when the answer needs primes above the bound."""
    if len(P) < k:
        # every omitted prime exceeds the sieve bound: bound any completion from below
        lb = math.prod(P) * (sieve_bound + 1) ** (k - len(P))
        if lb < U:
            raise SieveBoundError(f"D={D}: {len(P)} eligible primes below the sieve bound and a completion "
                                  "could stay below U; raise the sieve bound")
        return None
    Tk = math.prod(P[:k])
    if Tk >= U:
        return None
    cap = (U - 1) // (Tk // P[k - 1])
    if cap >= sieve_bound:
        raise SieveBoundError(f"D={D}: cap {cap} reaches the sieve bound; raise it")
    Pc = [q for q in P if q <= cap]
    rmax = 0
    for r in range(1, k + 1):
        if k + r > len(Pc):
            break
        num = Tk * math.prod(Pc[k:k + r])
        den = math.prod(P[k - r:k])
        if num // den < U:
            rmax = r
        else:
            break
    s = sum(1 for p in U_factors if D % (int(p) - 1) != 0)
    return {"D": D, "s": s, "pool": len(P), "cap": cap, "pool_capped": len(Pc), "rmax": rmax,
            "digits_T64": len(str(Tk))}


def divisor_family(U: int, U_factors, M: int | None = None, k: int = 64,
                   sieve_bound: int = SIEVE_BOUND) -> tuple[dict, list[dict]]:
    """Survivor rows of every divisor D of M = lambda(U) (the incumbent's own family), in divisor order.
    Returns (factorisation of M, rows)."""
    U = int(U)
    if M is None:
        M = carmichael_lambda(U_factors)
    lat = DivisorLattice(M, sieve_bound)
    order = sorted(range(len(lat.values)), key=lambda j: lat.values[j])
    rows = []
    for j in order:
        row = census_row(lat.values[j], lat.pool(j), U, U_factors, k, sieve_bound)
        if row is not None:
            rows.append(row)
    return dict(lat.fm), rows


def family_instances(rows, U: int, r_min: int = 1, r_max: int | None = None, k: int = 64,
                     sieve_bound: int = SIEVE_BOUND, with_base: bool = True):
    """(row, radius, Instance) for every survivor row: radius 0 (the k smallest primes themselves, when
    with_base) and radii r_min..min(rmax, r_max), each over the full capped pool with bound n < U -- the
    per-family runs of gpu/run_mstar_family.py:66-94, here as one portfolio.  Rows whose modulus has an
    odd part of 2^63 or more, or a 2-adic part above 2^32, are skipped (the reference skips every
    modulus of 2^64 or more)."""
    from .solve import Instance
    out = []
    pools = _Pools([int(r["D"]) for r in rows if _searchable(int(r["D"]))], sieve_bound)
    for row in rows:
        D, cap, rmax = int(row["D"]), int(row["cap"]), int(row["rmax"])
        if not _searchable(D):
            continue
        P = pools(D)
        Pc = [q for q in P if q <= cap]
        if len(Pc) != int(row["pool_capped"]):
            raise ValueError(f"D={D}: capped pool has {len(Pc)} primes, the row says {row['pool_capped']}")
        base = Pc[:k]
        hi = min(rmax, 10 if r_max is None else r_max, 10)      # instances hold radii up to 10
        radii = ([0] if with_base else []) + list(range(max(1, r_min), hi + 1))
        for r in radii:
            out.append((row, r, Instance.build(D, Pc, base, r, U - 1)))
    return out


def _searchable(D: int) -> bool:
    """Moduli the joins take: odd part below 2^63 and 2-adic part at most 2^32 (D may be 2^64 or
    more: keys are then taken mod 2^64 and matches confirmed exactly)."""
    a = (D & -D).bit_length() - 1
    return D >= 2 and (D >> a) < 1 << 63 and a <= 32


def _top_index(D: int) -> int:
    """Index of D itself among the divisors of D (the last exponent vector of the lattice)."""
    fm = factorize(D)
    return math.prod(e + 1 for e in fm.values()) - 1


class _Pools:
    """Eligible pools of the rows' moduli from one lattice of their lcm (every row of one family
    divides lambda), or one lattice per modulus when the lcm has too many divisors."""

    def __init__(self, Ds, sieve_bound: int, max_divisors: int = 1 << 20):
        self.sieve_bound = sieve_bound
        self.lat = None
        L = math.lcm(*[int(D) for D in Ds]) if Ds else 1
        if math.prod(e + 1 for e in factorize(L).values()) <= max_divisors:
            self.lat = DivisorLattice(L, sieve_bound)

    def __call__(self, D: int) -> list[int]:
        if self.lat is not None:
            return self.lat.pool(self.lat.index[int(D)])
        return DivisorLattice(D, self.sieve_bound).pool(_top_index(D))


def family_run(rows, U: int, r_min: int = 1, r_max: int | None = None, split: int = 4000, k: int = 64,
               sieve_bound: int = SIEVE_BOUND, consider=None, log=None, solver=None, workers: int = 2) -> dict:
    """Run every survivor row as gpu/run_mstar_family.py:66-94 drives the reference's GPU driver: the
    k smallest primes of the capped pool checked as a Carmichael number below U (radius 0), then each
    radius r_min..min(rmax, r_max) at the driver's h-stratum bound, through ``driver.run_instance`` (the
    driver's Icap/Dmin/affordable-pool bounds, product-bounded producers and record join on the GPU).
    Radii 1..16 are run; radii whose bounds need more than 128-bit products (or colex ids of 2^64 and
    more) are reported as skipped.

    With workers > 1 the instances' GPU joins run ahead on that many worker threads, each with its own
    solver and CUDA stream (one instance's kernels overlap another's host work), while the exact
    checks, consider() and log() run here in the order above, exactly as with one worker.

    Returns (runs, completions): runs = {D: {"base_carmichael", "base_below_U", "instances": [per-radius
    counts], "skipped": [r]}}; completions = the (key, factors, label) of every completion below U that
    was given to consider(key, factors, label) (the default consider only collects them)."""
    from . import bsolve, driver
    from .certify import verify_certificate
    from .solve import Solver, Tuning
    hits = []
    user = consider

    def consider(key, fac, label):
        hits.append((key, tuple(fac), label))
        return user(key, fac, label) if user is not None else True
    solver = solver or Solver(tuning=Tuning(strategy="bounded"))
    out = {}
    pools = _Pools([int(r["D"]) for r in rows if _searchable(int(r["D"]))], sieve_bound)
    # host pass: every row's base and the instances to join, in the reference's order
    steps = []                     # ("base", D, base) or ("inst", rec, (base, INS, r, h, D))
    for row in rows:
        D, cap, rmax = int(row["D"]), int(row["cap"]), int(row["rmax"])
        if not _searchable(D):
            out[D] = {"unsupported": "odd part of 2^63 or more, or 2-adic part above 2^32"}
            continue
        P = pools(D)
        Pc = [q for q in P if q <= cap]
        base, INS = Pc[:k], Pc[k:]
        ok, n, _ = verify_certificate(base)
        rec = {"base_carmichael": bool(ok), "base_below_U": bool(ok and n < U), "instances": [], "skipped": []}
        if ok and n < U:
            steps.append(("base", D, base))
        hi = rmax if r_max is None else min(rmax, r_max)
        for r in range(max(1, r_min), hi + 1):
            h = driver.hmax_for(base, INS, r, U, split)
            if h < 0:
                continue
            Icap, _Dmin, _cap_r, aff = driver.instance_bounds(base, INS, r, U)
            if len(aff) >= r and not bsolve.bounds_fit(base, aff, r, Icap):
                rec["skipped"].append(r)
                continue
            steps.append(("inst", rec, (base, INS, r, h, D)))
        out[D] = rec
    jobs = [a for kind, _, a in steps if kind == "inst"]
    joined = _join_ahead(jobs, U, split, solver, workers)
    for kind, x, a in steps:
        if kind == "base":
            consider((x, "ksmall", 0, 0), a, "census_base")
            continue
        base, INS, r, h, D = a
        st: dict = {}
        driver.run_instance("ksmall", base, INS, r, h, D, U, split, consider, log, st, solver,
                            joined=next(joined))
        x["instances"].append(st["last"])
    return out, hits


def _join_ahead(jobs, U: int, split: int, solver, workers: int):
    """Iterator over driver.instance_join's results for jobs (base, INS, r, h, M), in order.  With
    workers > 1 the joins run on worker threads, each with a solver on its own CUDA stream (the
    library's C calls release the interpreter lock while they wait for the device)."""
    from . import driver
    if workers <= 1 or len(jobs) < 2:
        for base, INS, r, h, M in jobs:
            yield driver.instance_join(base, INS, r, h, M, U, split, solver)
        return
    import queue
    import threading
    from concurrent.futures import ThreadPoolExecutor

    import torch

    from .solve import Solver
    # the worker solvers live on the caller's solver, so later runs reuse their streams and buffers
    ws = getattr(solver, "_join_workers", None)
    if ws is None or len(ws) < workers:
        ws = solver._join_workers = [Solver(solver.device, stream=torch.cuda.Stream(solver.device),
                                            tuning=solver.tuning) for _ in range(workers)]
    free: queue.Queue = queue.Queue()
    for w in ws[:workers]:
        free.put(w)
    local = threading.local()

    def run(job):
        if getattr(local, "solver", None) is None:
            local.solver = free.get()
        base, INS, r, h, M = job
        return driver.instance_join(base, INS, r, h, M, U, split, local.solver)

    with ThreadPoolExecutor(max_workers=workers) as ex:
        futs = [ex.submit(run, j) for j in jobs]
        for f in futs:
            yield f.result()


# -- lambda-neighbourhood census ------------------------------------------------------------

# The two moduli of the reference's exclusion theorems: every 64-factor Carmichael number below the
# record N has a prime q with (q-1) not dividing M0 and a prime q' with (q'-1) not dividing lambda(N)
# (gpu/lambda_neighbourhood.py:61, 78-79).
WITNESS_M0 = 1768248177696000
WITNESS_LN = 155016423578016000


def two_witness_min(P, U: int, M0: int = WITNESS_M0, LN: int = WITNESS_LN, k: int = 64):
    """Smallest k-product from the ascending pool P that contains a prime q with (q-1) not dividing M0
    and a prime q' with (q'-1) not dividing LN (one prime may be both), or None when none exists
    (gpu/lambda_neighbourhood.py:78-97)."""
    def fill(req):
        rest = [q for q in P if q not in req]
        if len(rest) < k - len(req):
            return None
        return math.prod(req + rest[:k - len(req)])

    best = None
    both = [q for q in P if M0 % (q - 1) and LN % (q - 1)]
    if both:
        v = fill([both[0]])
        best = v if best is None or (v is not None and v < best) else best
    only0 = [q for q in P if M0 % (q - 1) and LN % (q - 1) == 0]
    onlyN = [q for q in P if LN % (q - 1) and M0 % (q - 1) == 0]
    if only0 and onlyN:
        v = fill(sorted([only0[0], onlyN[0]]))
        best = v if best is None or (v is not None and v < best) else best
    return best


class _Candidates:
    """Primes q <= bound with (q-1) dividing L, with the exponent vectors of q-1 over L's primes, for
    the pools of the divisors of L: relaxed pool of D = {q : (q-1) | D}, pool Q(D) = relaxed pool
    minus the primes dividing D."""

    def __init__(self, L_fm: dict, sieve_bound: int):
        self.primes = sorted(L_fm)
        isp = _is_prime_table(sieve_bound)
        qs, vecs = [], []

        def walk(i, d, vec):                      # divisors of L up to the bound only
            if i == len(self.primes):
                if 3 <= d + 1 <= sieve_bound and isp[d + 1]:
                    qs.append(d + 1)
                    vecs.append(tuple(vec))
                return
            p = self.primes[i]
            for e in range(L_fm[p] + 1):
                if d * p ** e > sieve_bound:
                    break
                vec.append(e)
                walk(i + 1, d * p ** e, vec)
                vec.pop()
        walk(0, 1, [])
        order = sorted(range(len(qs)), key=lambda j: qs[j])
        self.q = np.asarray([qs[j] for j in order], dtype=np.int64)
        self.E = np.asarray([vecs[j] for j in order], dtype=np.int16).reshape(len(order), len(self.primes))
        self.pidx = np.asarray([self.primes.index(int(q)) if int(q) in L_fm else -1 for q in self.q],
                               dtype=np.int64)

    def pools(self, e) -> tuple[list[int], list[int]]:
        """(relaxed pool, pool) of the divisor with exponent vector e (over L's primes)."""
        e = np.asarray(e, dtype=np.int16)
        ok = (self.E <= e).all(axis=1)
        inL = self.pidx >= 0
        divides = np.zeros(len(self.q), dtype=bool)
        divides[inL] = e[self.pidx[inL]] >= 1
        return [int(x) for x in self.q[ok]], [int(x) for x in self.q[ok & ~divides]]


def _relaxed_survives(Pr, U, k, sieve_bound, M0, LN) -> bool:
    """False only when even the relaxed pool cannot give a qualifying k-product below U; both tests are
    monotone in D over the relaxed pool, so pruning on them is sound (gpu/lambda_neighbourhood.py:62-77)."""
    if len(Pr) < k:
        return math.prod(Pr) * (sieve_bound + 1) ** (k - len(Pr)) < U
    if math.prod(Pr[:k]) >= U:
        return False
    w = two_witness_min(Pr, U, M0, LN, k)
    return w is not None and w < U


def _neighbour_job(seed: int, p: int, U: int, U_factors, k: int, sieve_bound: int, M0: int, LN: int):
    """Rows of the new moduli D | (seed or seed*q) * p with p | D, as gpu/lambda_neighbourhood.py:99-149:
    a top-down walk over exponent vectors (p's exponent fixed at 1) from each neighbour, pruned where the
    relaxed pool fails, sharing visits between the neighbours of one (seed, p)."""
    sfm = factorize(seed)
    if seed % p == 0:
        return {}, []
    L_fm = {q: e + 1 for q, e in sfm.items()}
    L_fm[p] = 1
    cand = _Candidates(L_fm, sieve_bound)
    col = {q: i for i, q in enumerate(cand.primes)}
    variants = [(None, 0, dict(sfm))] + [(q, -1, {**sfm, q: e + 1}) for q, e in sfm.items()]
    seen: dict = {}
    rows: dict = {}
    problems: list = []
    for q, j, fm in variants:
        primes = [x for x in fm if x != p]
        emax = [fm[x] for x in primes]
        out = []
        stack = [list(emax)]

        def visit(vec):
            D = p * math.prod(x ** e for x, e in zip(primes, vec))
            if D in seen:
                return False
            e_full = [0] * len(cand.primes)
            for x, ex in zip(primes, vec):
                e_full[col[x]] = ex
            e_full[col[p]] = 1
            relaxed, pool = cand.pools(e_full)
            if not _relaxed_survives(relaxed, U, k, sieve_bound, M0, LN):
                seen[D] = False
                return False
            seen[D] = True
            try:
                row = census_row(D, pool, U, U_factors, k, sieve_bound)
            except SieveBoundError:
                problems.append(("SIEVE", D))
                row = None
            if row is not None:
                out.append(row)
            return True

        # depth-first in the reference's order: a node, then its children by decrementing each exponent
        def rec(vec):
            if not visit(vec):
                return
            for i in range(len(vec)):
                if vec[i] > 0:
                    v2 = list(vec)
                    v2[i] -= 1
                    rec(v2)
        rec(list(emax))
        for r in out:
            if r["D"] not in rows:
                rows[r["D"]] = dict(r, seed=str(seed), q=q, j=j, p=p)
    return rows, problems


def _neighbour_job_star(args):
    return _neighbour_job(*args)


def lambda_neighbourhood(seeds, pmax: int, U: int, U_factors, k: int = 64, sieve_bound: int = SIEVE_BOUND,
                         M0: int = WITNESS_M0, LN: int = WITNESS_LN, procs: int = 1) -> tuple[list[dict], list]:
    """New candidate moduli one step from the seed moduli (gpu/lambda_neighbourhood.py:151-188): for every
    seed M and prime 3 <= p <= pmax not dividing M, the divisors D of M*p and of M*q*p (q a prime of M)
    with p | D that can carry a k-factor Carmichael number below U, kept when their cheapest k-product
    with both exclusion witnesses is below U.  Returns (rows sorted richest first, sieve problems)."""
    isp = _is_prime_table(max(pmax, 3))
    primes = [q for q in range(3, pmax + 1) if isp[q]]
    seeds = [int(m) for m in seeds]
    jobs = [(M, q, int(U), list(U_factors), k, sieve_bound, M0, LN) for M in seeds for q in primes]
    covered = set()
    for M in seeds:
        covered.update(DivisorLattice(M, sieve_bound).values)
    results = []
    if procs > 1:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(procs) as pool:
            results = pool.map(_neighbour_job_star, jobs, chunksize=1)
    else:
        results = [_neighbour_job(*a) for a in jobs]
    rows: dict = {}
    problems: list = []
    for r, pr in results:                      # job order (the reference keeps the first to finish)
        problems += pr
        for D, row in r.items():
            if D in covered:
                continue
            if D not in rows or row["digits_T64"] < rows[D]["digits_T64"]:
                rows[D] = row
    kept = []
    for row in rows.values():
        D = row["D"]
        lat = _Candidates({**factorize(D)}, sieve_bound)
        _, pool = lat.pools([factorize(D)[x] for x in lat.primes])
        w = two_witness_min([q for q in pool if q <= row["cap"]], U, M0, LN, k)
        if w is None or w >= U:
            continue
        kept.append(dict(row, w2_digits=len(str(w))))
    kept.sort(key=lambda r: (r["w2_digits"], r["digits_T64"], -r["rmax"], r["D"]))
    return kept, problems

