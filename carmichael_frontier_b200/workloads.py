"""Seeded synthetic instances with the shapes of the k=64 search's benchmark configurations.

No public dataset is involved: moduli are drawn from a seeded PRNG with the
distribution the benchmark configurations state, and pools are the eligible
primes Q(M) = {q prime : (q-1) | M, q does not divide M}
(gpu/mitm_gpu_mstar_driver.py:77-82 builds the same pool by trial division).
"""
from __future__ import annotations

import math
import random
from dataclasses import dataclass

from .certify import is_probable_prime

MID_PRIMES = (11, 13, 17, 19, 23, 29, 31, 37, 41, 43)


@dataclass(frozen=True)
class Workload:
    """One solve request: solve(M, Q, B0, r, B)."""
    name: str
    M: int
    Q: tuple[int, ...]
    B0: tuple[int, ...]
    r: int
    B: int

    @property
    def INS(self) -> tuple[int, ...]:
        b = set(self.B0)
        return tuple(q for q in self.Q if q not in b)

    @property
    def n_D(self) -> int:
        return math.comb(len(self.B0), self.r)

    @property
    def n_I(self) -> int:
        return math.comb(len(self.INS), self.r)


def _factor_small(M: int) -> dict[int, int] | None:
    f, m, p = {}, M, 2
    while p * p <= m and p < 1 << 20:
        while m % p == 0:
            f[p] = f.get(p, 0) + 1
            m //= p
        p += 1 if p == 2 else 2
    if m > 1:
        if m >= 1 << 40 and not is_probable_prime(m):
            return None
        f[m] = f.get(m, 0) + 1
    return f


def divisors(M: int) -> list[int] | None:
    f = _factor_small(M)
    if f is None:
        return None
    ds = [1]
    for p, e in f.items():
        ds = [d * p ** k for d in ds for k in range(e + 1)]
    return sorted(ds)


def eligible_pool(M: int, cap: int | None = None, nmax: int | None = None) -> list[int]:
    """Q(M), ascending: primes q <= cap (all, when cap is None) with (q-1) | M and q not dividing M."""
    ds = divisors(M)
    if ds is not None:
        out = [d + 1 for d in ds if d + 1 > 2 and (cap is None or d + 1 <= cap)
               and M % (d + 1) != 0 and is_probable_prime(d + 1)]
    else:
        if cap is None:
            raise ValueError("M has a large composite cofactor: give a prime cap")
        out = [q for q in range(3, cap + 1, 2) if M % (q - 1) == 0 and M % q != 0 and is_probable_prime(q)]
    out.sort()
    return out[:nmax] if nmax is not None else out


def draw_modulus(seed: int) -> int:
    """M = 2^a 3^b 5^c 7^d * (4-6 distinct primes from 11..43), redrawn until 10^15 <= M < 2^62."""
    rng = random.Random(seed)
    while True:
        a = rng.randint(5, 9)
        b = rng.randint(2, 5)
        c = rng.randint(1, 3)
        d = rng.randint(0, 2)
        mids = rng.sample(MID_PRIMES, rng.randint(4, 6))
        M = 2 ** a * 3 ** b * 5 ** c * 7 ** d
        for p in mids:
            M *= p
        if 10 ** 15 <= M < 2 ** 62:
            return M


def product(xs) -> int:
    out = 1
    for x in xs:
        out *= x
    return out


def config1() -> Workload:
    """k=29, M = 21621600, Q(M) complete, B0 = 29 smallest, r = 2, B = prod(B0) * 10^8."""
    M = 21621600
    Q = eligible_pool(M)
    B0 = Q[:29]
    return Workload("k29_M21621600_r2", M, tuple(Q), tuple(B0), 2, product(B0) * 10 ** 8)


def config2(seed: int, r: int = 5, B: int = 10 ** 148) -> Workload | None:
    """k=64 single modulus: seeded M, Q(M) = primes <= 5518 (cap 320), B0 = 64 smallest."""
    M = draw_modulus(seed)
    Q = eligible_pool(M, 5518, 320)
    if len(Q) < 64 + r:
        return None
    return Workload(f"k64_seed{seed}_r{r}", M, tuple(Q), tuple(Q[:64]), r, B)


def config2_seeds(count: int, start: int = 0, r: int = 5) -> list[Workload]:
    out, s = [], start
    while len(out) < count:
        w = config2(s, r)
        if w is not None:
            out.append(w)
        s += 1
    return out


def config3(count: int = 1024, seed: int = 0) -> list[Workload]:
    """Portfolio: seeded moduli, pool size uniform in 120..400 from primes < 10^5 (truncated),
    radius uniform in {4, 5, 6}, B = 10^148; moduli whose pool is too small are redrawn."""
    rng = random.Random(10_000 + seed)
    out, s = [], 0
    while len(out) < count:
        M = draw_modulus(1_000_000 * (seed + 1) + s)
        s += 1
        size = rng.randint(120, 400)
        r = rng.choice((4, 5, 6))
        Q = eligible_pool(M, 10 ** 5)
        if len(Q) < size:
            continue
        Q = Q[:size]
        out.append(Workload(f"portfolio{len(out)}_r{r}_n{size}", M, tuple(Q), tuple(Q[:64]), r, 10 ** 148))
    return out


def config4(seed: int = 0, r: int = 7) -> Workload:
    """Large radius: seeded M, pool capped at 160 primes (|INS| = 96), r = 7."""
    s = seed
    while True:
        M = draw_modulus(s)
        Q = eligible_pool(M, 10 ** 5, 160)
        if len(Q) == 160:
            return Workload(f"k64_large_seed{s}_r{r}", M, tuple(Q), tuple(Q[:64]), r, 10 ** 148)
        s += 1


def config5_requests(count: int = 10_000, seed: int = 0) -> list[Workload]:
    """Serving stream: k uniform in 64..100, pool 80..320 (>= k + r), r in 3..6, B = prod(B0) * 10^4."""
    rng = random.Random(20_000 + seed)
    out, s = [], 0
    while len(out) < count:
        M = draw_modulus(2_000_000 * (seed + 1) + s)
        s += 1
        k = rng.randint(64, 100)
        r = rng.randint(3, 6)
        size = rng.randint(80, 320)
        Q = eligible_pool(M, 10 ** 5)
        if len(Q) < max(size, k + r):
            continue
        Q = Q[:max(size, k + r)]
        B0 = Q[:k]
        out.append(Workload(f"req{len(out)}_k{k}_r{r}", M, tuple(Q), tuple(B0), r, product(B0) * 10 ** 4))
    return out
