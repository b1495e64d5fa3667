"""RNS parameter helpers for building workloads: NTT-friendly primes
(q = 1 mod 2N) and primitive 2N-th roots of unity.

The search is deterministic (no random state), in the manner of the
reference test suite's generators (tests/common/parameters.hpp:58-122): the
largest prime of the form k*2N + 1 at or below a position inside
[2^(bits-1), 2^bits), then upward if none.  Miller-Rabin with the
deterministic 64-bit base set.
"""
from __future__ import annotations

_BASES = (2, 325, 9375, 28178, 450775, 9780504, 1795265022)
_SMALL = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)


def is_prime(n: int) -> bool:
    if n < 2:
        return False
    for p in _SMALL:
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in _BASES:
        if a % n == 0:
            continue
        x = pow(a % n, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def ntt_prime_near(degree: int, bits: int, num: int = 1, den: int = 1) -> int:
    """Prime q = 1 mod 2*degree with bit width `bits`, nearest at or below
    lo + (hi - lo) * num / den, else the nearest above it."""
    if not (2 <= bits < 63) or den == 0 or num > den:
        raise ValueError("bad prime request")
    step = 2 * degree
    lo, hi = 1 << (bits - 1), (1 << bits) - 1
    target = lo + (hi - lo) * num // den
    q = target - ((target - 1) % step)
    while q >= lo and q > step:
        if is_prime(q):
            return q
        q -= step
    q = target - ((target - 1) % step)
    if q < target:
        q += step
    while q <= hi:
        if is_prime(q):
            return q
        q += step
    raise ValueError("no NTT-friendly prime of that width")


def primitive_root(degree: int, q: int) -> int:
    """Smallest-generator primitive 2*degree-th root of unity mod q."""
    order = 2 * degree
    e = (q - 1) // order
    for a in range(2, 100000):
        psi = pow(a, e, q)
        if psi != 1 and pow(psi, degree, q) == q - 1:
            return psi
    raise ValueError("no primitive root found")


def rns_moduli(degree: int, count: int, bits_lo: int, bits_hi: int):
    """`count` distinct NTT-friendly primes cycling through widths
    bits_lo..bits_hi, at positions 1/4, 2/4, 3/4 of each width."""
    widths = list(range(bits_lo, bits_hi + 1))
    out, seen = [], set()
    i = 0
    while len(out) < count:
        bits = widths[i % len(widths)]
        pos = 1 + (i // len(widths)) % 3
        q = ntt_prime_near(degree, bits, pos, 4)
        if q not in seen:
            seen.add(q)
            out.append((q, primitive_root(degree, q)))
        i += 1
        if i > 100 * count:
            raise ValueError("not enough distinct primes")
    return out
