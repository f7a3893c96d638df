"""Standalone witness verifier (mirrors review/verify_cube.py:8-20).

Deliberately independent of the focus geometry, the tables and the GPU code: its own prime list,
bisection cube root and exponent tests.  ``verify_many`` evaluates the same predicate for many
values at once (the parallel CPU verification a small prime bound needs, where a batch emits
millions of survivors) and gives the same rows.
"""
from __future__ import annotations

from collections.abc import Sequence
from math import isqrt
from typing import Any

import numpy as np


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


# ------------------------------------------------------------------------------------------
# Many values at once.  The same predicate, evaluated column-wise on 64-bit limbs with numpy
# (values below 2^96, as every output of the sieve is), in chunks on a thread pool (numpy releases
# the interpreter lock inside its array operations).

VECTOR_MIN = 2048          # fewer values: verify() one by one
MATERIALISE_MAX = 1 << 20  # more non-cubes than this: the rows are built when read


def _mod(lo: np.ndarray, hi: np.ndarray, q: int) -> np.ndarray:
    """x mod q for x = hi 2^64 + lo, hi < 2^32, exactly in uint64 arithmetic."""
    return ((hi % np.uint64(q)) * np.uint64((1 << 64) % q) + lo % np.uint64(q)) % np.uint64(q)


def cube_limbs(a: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """a^3 as (high, low) 64-bit limbs for a < 2^32."""
    sq = a * a                                           # < 2^64
    h, l = sq >> np.uint64(32), sq & np.uint64(0xFFFFFFFF)
    ha, la = h * a, l * a                                # a^3 = ha 2^32 + la, each < 2^64
    low = (ha << np.uint64(32)) + la
    return (ha >> np.uint64(32)) + (low < la).astype(np.uint64), low


def _le(h1: np.ndarray, l1: np.ndarray, h2: np.ndarray, l2: np.ndarray) -> np.ndarray:
    return (h1 < h2) | ((h1 == h2) & (l1 <= l2))


def icbrt_many(lo: np.ndarray, hi: np.ndarray) -> np.ndarray:
    """Floor cube roots of x = hi 2^64 + lo < 2^96: a double estimate (within one of the root),
    corrected exactly in 128-bit limbs."""
    xf = hi.astype(np.float64) * 18446744073709551616.0 + lo.astype(np.float64)
    a = np.floor(np.cbrt(xf)).astype(np.int64)
    a = np.clip(a, 0, (1 << 32) - 2).astype(np.uint64)
    for _ in range(2):                                   # a^3 > x: step down
        h, l = cube_limbs(a)
        a = np.where(_le(h, l, hi, lo) | (a == 0), a, a - np.uint64(1))
    top = np.uint64((1 << 32) - 1)                       # the root of any x < 2^96
    for _ in range(2):                                   # (a + 1)^3 <= x: step up
        h, l = cube_limbs(np.minimum(a + np.uint64(1), top))
        a = np.where((a < top) & _le(h, l, hi, lo), a + np.uint64(1), a)
    return a


class Witnesses(Sequence):
    """verify() rows of the non-cubes among many values, computed column-wise; a row is the same
    dict verify(n, p) returns and is built when it is read."""

    def __init__(self, p: int, lo: np.ndarray, hi: np.ndarray, root: np.ndarray, valid: np.ndarray,
                 failing: dict[int, list[int]]) -> None:
        self.p, self.lo, self.hi, self.root, self.valid, self.failing = p, lo, hi, root, valid, failing

    def __len__(self) -> int:
        return len(self.lo)

    def row(self, i: int) -> dict[str, Any]:
        n = int(self.hi[i]) << 64 | int(self.lo[i])
        return dict(n=str(n), p=self.p, cube_root_floor=str(int(self.root[i])), perfect_cube=False,
                    failing_primes=list(self.failing.get(i, [])), valid_pseudocube=bool(self.valid[i]),
                    claim='Candidate validity only; no minimality claim.')

    def __getitem__(self, i):
        if isinstance(i, slice):
            return [self.row(k) for k in range(*i.indices(len(self)))]
        if i < 0:
            i += len(self)
        if not 0 <= i < len(self):
            raise IndexError(i)
        return self.row(i)

    def __eq__(self, other: object) -> bool:
        return isinstance(other, Sequence) and len(other) == len(self) and all(a == b for a, b in zip(self, other))

    @property
    def all_valid(self) -> bool:
        return bool(self.valid.all())


def _columns(lo: np.ndarray, hi: np.ndarray, p: int, primes: tuple[int, ...],
             tables: dict[int, np.ndarray]) -> tuple[np.ndarray, np.ndarray, np.ndarray, dict[int, list[int]]]:
    """Per value: the local test (n > 0, n = +-1 mod 9, no failing prime), the floor cube root, the
    perfect-cube flag, and the failing primes of the values that have any."""
    ok = np.isin(_mod(lo, hi, 9), np.array([1, 8], dtype=np.uint64)) & ((lo != 0) | (hi != 0))
    failing: dict[int, list[int]] = {}
    for q in primes:
        r = _mod(lo, hi, q).astype(np.int64)
        bad = tables[q][r]                               # r = 0, or not a cubic residue when q = 1 mod 3
        if bad.any():
            for i in np.nonzero(bad)[0].tolist():
                failing.setdefault(i, []).append(q)
            ok &= ~bad
    root = icbrt_many(lo, hi)
    h, l = cube_limbs(root)
    cube = (h == hi) & (l == lo)
    return ok, root, cube, failing


def verify_many(lo: np.ndarray, hi: np.ndarray, p: int, threads: int | None = None) -> tuple[np.ndarray, np.ndarray, Witnesses]:
    """Column-wise verify() of many values x = hi 2^64 + lo < 2^96.  Returns the local test per value
    (local3), the perfect-cube flags, and the verify() rows of the non-cubes in input order."""
    import os
    from concurrent.futures import ThreadPoolExecutor
    primes = tuple(q for q in range(2, p + 1) if all(q % d for d in range(2, isqrt(q) + 1)))
    if p not in primes or p % 3 != 1:
        raise ValueError('invalid prime cutoff')
    lo = np.ascontiguousarray(lo, dtype=np.uint64)
    hi = np.ascontiguousarray(hi, dtype=np.uint64)
    if len(hi) and int(hi.max()) >> 32:
        raise ValueError('values must be below 2^96')
    tables = {}
    for q in primes:                                     # failure table of verify(): r = 0, or r^((q-1)/3) != 1
        tables[q] = np.array([r == 0 or (q % 3 == 1 and pow(r, (q - 1) // 3, q) != 1) for r in range(q)], dtype=bool)
    n = len(lo)
    step = max(1 << 16, -(-n // (4 * (threads or os.cpu_count() or 1))))
    spans = [(a, min(n, a + step)) for a in range(0, n, step)] or [(0, 0)]
    with ThreadPoolExecutor(max_workers=threads or os.cpu_count() or 1) as pool:
        parts = list(pool.map(lambda s: _columns(lo[s[0]:s[1]], hi[s[0]:s[1]], p, primes, tables), spans))
    ok = np.concatenate([part[0] for part in parts])
    root = np.concatenate([part[1] for part in parts])
    cube = np.concatenate([part[2] for part in parts])
    failing: dict[int, list[int]] = {}
    for (a, _), part in zip(spans, parts):
        for i, qs in part[3].items():
            failing[a + i] = qs
    keep = np.nonzero(~cube)[0]
    renumber = {int(j): k for k, j in enumerate(keep.tolist())} if failing else {}
    witnesses = Witnesses(p, lo[keep], hi[keep], root[keep], ok[keep],
                          {renumber[i]: qs for i, qs in failing.items() if i in renumber})
    return ok, cube, witnesses
