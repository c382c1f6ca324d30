"""Certificate check of a claimed Carmichael factorisation (host, exact integers).

Same decision as the reference's frozen checker ref/ref_carmichael.py:55-72:
at least 3 factors, pairwise distinct, each prime by a strong-probable-prime
test to the first twelve prime bases (deterministic below 3.3e24 and far
beyond the pool primes used here), and Korselt's criterion (p-1) | (n-1) for
every factor.  Every hit returned by ``solve`` passes through it.
"""
from __future__ import annotations

_BASES = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)


def is_probable_prime(n: int) -> bool:
    if n < 2:
        return False
    for b in _BASES:
        if n % b == 0:
            return n == b
    d, s = n - 1, 0
    while not d & 1:
        d >>= 1
        s += 1
    for b in _BASES:
        x = pow(b, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def verify_certificate(primes) -> tuple[bool, int, str]:
    """(ok, n, reason) for n = prod(primes) being Carmichael with exactly len(primes) factors."""
    ps = [int(p) for p in primes]
    if len(ps) < 3:
        return False, 0, "fewer than 3 prime factors"
    if len(set(ps)) != len(ps):
        return False, 0, "repeated factor (n not squarefree)"
    for p in ps:
        if not is_probable_prime(p):
            return False, 0, f"factor {p} is not prime"
    n = 1
    for p in ps:
        n *= p
    for p in ps:
        if (n - 1) % (p - 1):
            return False, n, f"Korselt fails at p={p}"
    return True, n, f"Carmichael with exactly {len(ps)} prime factors"
