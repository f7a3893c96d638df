"""Residue tables of the local pseudocube conditions (mirrors pseudocube/tables.py:9-36).

Allowed residues: {1, 8} mod 9; the nonzero cubes mod q for q = 1 (mod 3); every nonzero residue
mod any other prime.  Tables come from cubing, independently of the exponent test in
``predicate.local3``.
"""
from __future__ import annotations

import hashlib
import json
from functools import lru_cache
from math import isqrt
from typing import Any


def sieve_primes(p: int) -> list[int]:
    """Primes <= p by Eratosthenes (pseudocube/tables.py:9-15)."""
    if p < 2:
        return []
    composite = bytearray(p + 1)
    for q in range(2, isqrt(p) + 1):
        if not composite[q]:
            composite[q * q::q] = b'\x01' * len(range(q * q, p + 1, q))
    return [q for q in range(2, p + 1) if not composite[q]]


@lru_cache(maxsize=None)
def allowed(q: int) -> tuple[int, ...]:
    """Allowed residues mod q (pseudocube/tables.py:18-23)."""
    if q == 9:
        return (1, 8)
    if q % 3 == 1:
        return tuple(sorted({pow(a, 3, q) for a in range(1, q)}))
    return tuple(range(1, q))


def packed(q: int) -> list[int]:
    """32-bit bitmap words of allowed(q) (pseudocube/tables.py:26-30)."""
    words = [0] * ((q + 31) // 32)
    for a in allowed(q):
        words[a >> 5] |= 1 << (a & 31)
    return words


def definition(p: int) -> dict[str, Any]:
    """Table set and its hash (pseudocube/tables.py:33-36)."""
    tables = {str(q): list(allowed(q)) for q in (9, *sieve_primes(p)) if q != 3}
    raw = json.dumps(tables, sort_keys=True, separators=(',', ':')).encode()
    return {'tables': tables, 'sha256': hashlib.sha256(raw).hexdigest()}
