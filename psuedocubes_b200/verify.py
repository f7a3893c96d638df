"""Standalone witness verifier (mirrors review/verify_cube.py:8-20).

Deliberately independent of the focus geometry, the tables and the GPU code: its own prime list,
bisection cube root and exponent tests.
"""
from __future__ import annotations

from math import isqrt
from typing import Any


def verify(n: int, p: int) -> dict[str, Any]:
    primes = [q for q in range(2, p + 1) if all(q % d for d in range(2, isqrt(q) + 1))]
    if p not in primes or p % 3 != 1:
        raise ValueError('invalid prime cutoff')
    if n < 0:
        raise ValueError('negative integer')
    low, high = 0, n + 1
    while high - low > 1:
        middle = (low + high) // 2
        if middle * middle * middle <= n:
            low = middle
        else:
            high = middle
    failures = [q for q in primes if n % q == 0 or (q % 3 == 1 and pow(n, (q - 1) // 3, q) != 1)]
    cube = low ** 3 == n
    valid = n > 0 and n % 9 in (1, 8) and not failures and not cube
    return dict(n=str(n), p=p, cube_root_floor=str(low), perfect_cube=cube, failing_primes=failures,
                valid_pseudocube=valid, claim='Candidate validity only; no minimality claim.')
