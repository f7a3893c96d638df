"""Exact local predicate used to re-check every emitted value on the host.

Mirrors pseudocube/oracle.py:7-45 (primes_upto, validate_p, icbrt, is_perfect_cube, local3,
qualifies3).  This is the product's host verification step, not the test oracle.
"""
from __future__ import annotations

from functools import lru_cache
from math import isqrt


@lru_cache(maxsize=128)
def primes_upto(p: int) -> tuple[int, ...]:
    if type(p) is not int or p < 0:
        raise ValueError('prime limit must be a nonnegative integer')
    return tuple(q for q in range(2, p + 1) if all(q % d for d in range(2, isqrt(q) + 1)))


def validate_p(p: int) -> None:
    if type(p) is not int or p < 7 or p % 3 != 1 or p not in primes_upto(p):
        raise ValueError('p must be a prime congruent to 1 modulo 3')


def icbrt(n: int) -> int:
    """Floor cube root by bisection."""
    if type(n) is not int or n < 0:
        raise ValueError('cube root requires a nonnegative integer')
    lo, hi = 0, 1 << ((n.bit_length() + 2) // 3)
    while lo < hi:
        mid = (lo + hi + 1) >> 1
        if mid * mid * mid <= n:
            lo = mid
        else:
            hi = mid - 1
    return lo


def is_perfect_cube(n: int) -> bool:
    return n >= 0 and icbrt(n) ** 3 == n


def local3(n: int, p: int) -> bool:
    """Positive, n = +-1 mod 9, coprime to every prime <= p, cubic residue mod every q = 1 mod 3."""
    validate_p(p)
    if type(n) is not int or n <= 0 or n % 9 not in (1, 8):
        return False
    for q in primes_upto(p):
        if n % q == 0:
            return False
        if q % 3 == 1 and pow(n, (q - 1) // 3, q) != 1:
            return False
    return True


def qualifies3(n: int, p: int) -> bool:
    return local3(n, p) and not is_perfect_cube(n)
