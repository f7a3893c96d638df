"""Genuine-cube control on the device.

The reference cross-checks its campaign with two host checkers that count the integers a in
[first, last] coprime to every prime <= p (review/cube_count.c:12-37, a byte-segment sieve;
review/cube_count_independent.c:9-34, an odd-only bit sieve), run over the cube roots of the whole
interval (1e27, 3e27] at p = 619 by tools/check_cpu.py:24-29, which requires 38,322,775.  Each such
a gives a cube a^3 that passes every residual filter of bound p, so the count over the roots of
(lo, hi] is exactly the number of genuine cubes a correct sieve of (lo, hi] must emit.

``count_roots`` / ``list_roots`` run the device sieve ``pc_cube_roots``; ``checker_record`` gives
the one-line JSON record of the reference checkers (roots as decimal strings, the count as a
string); ``genuine_cube_count`` maps an x interval (lo, hi] to its roots.  ``python -m
psuedocubes_b200.cubes FIRST LAST P [--list]`` is the command-line form of the checkers.
"""
from __future__ import annotations

import ctypes
import json
import sys
from typing import Any

import numpy as np

from .gpu import Runtime
from .predicate import icbrt

ROOT_MAX = (1 << 32) - 1
P_MAX = 2000
ALGORITHM = 'device-bit-segment'


def _check(first: int, last: int, p: int) -> None:
    if not (1 <= first <= last <= ROOT_MAX and 2 <= p <= P_MAX):
        raise ValueError('cube roots need 1 <= first <= last < 2^32 and 2 <= p <= 2000')


def count_roots(runtime: Runtime, first: int, last: int, p: int) -> int:
    """How many a in [first, last] are coprime to every prime <= p."""
    _check(first, last, p)
    count = ctypes.c_uint64()
    runtime.call(runtime.lib.pc_cube_roots(runtime.ctx, first, last, p, None, 0, ctypes.byref(count), None), 'cube roots')
    return count.value


def list_roots(runtime: Runtime, first: int, last: int, p: int, cap: int | None = None) -> np.ndarray:
    """The a in [first, last] coprime to every prime <= p, ascending (uint32).  More than ``cap``
    roots raise OverflowError; by default ``cap`` admits every root of the range."""
    _check(first, last, p)
    cap = last - first + 1 if cap is None else cap
    out = np.zeros(max(1, cap), dtype=np.uint32)
    count = ctypes.c_uint64()
    runtime.call(runtime.lib.pc_cube_roots(runtime.ctx, first, last, p, out.ctypes.data, cap, ctypes.byref(count), None),
                 'cube roots')
    return out[:count.value]


def root_bounds(lo: int, hi: int) -> tuple[int, int] | None:
    """Inclusive cube-root bounds of the cubes in (lo, hi], or None when there are none."""
    first, last = icbrt(max(lo, 0)) + 1, icbrt(max(hi, 0))
    return (first, last) if first <= last else None


def genuine_cube_count(runtime: Runtime, p: int, lo: int, hi: int) -> int:
    """Genuine cubes of (lo, hi] at bound p: the cubes a^3 there with a coprime to every prime <= p."""
    bounds = root_bounds(lo, hi)
    return count_roots(runtime, bounds[0], bounds[1], p) if bounds else 0


def checker_record(runtime: Runtime, first: int, last: int, p: int, listed: bool = False) -> dict[str, Any]:
    """The record the reference checkers print (review/cube_count.c:24,35-36), from the device."""
    row: dict[str, Any] = dict(algorithm=ALGORITHM, root_first=str(first), root_last=str(last), p=p)
    if listed:
        roots = list_roots(runtime, first, last, p)
        row['roots'] = [str(int(a)) for a in roots]
        count = len(roots)
    else:
        count = count_roots(runtime, first, last, p)
    row.update(count=str(count), working_bytes=0)
    return row


def main(argv: list[str]) -> int:
    """FIRST LAST P [--list]: exit status 2 on invalid arguments, as the reference checkers."""
    args = [a for a in argv if a != '--list']
    listed = len(args) != len(argv)
    try:
        if len(args) != 3 or any(not a.isdigit() for a in args):
            raise ValueError('usage: FIRST LAST P [--list]')
        first, last, p = (int(a) for a in args)
        _check(first, last, p)
        if listed and last - first > 100000:
            raise ValueError('--list covers at most 100001 roots')
    except ValueError as exc:
        sys.stderr.write(f'{exc}\n')
        return 2
    runtime = Runtime(float('inf'), 1 << 30)
    try:
        print(json.dumps(checker_record(runtime, first, last, p, listed), separators=(',', ':')))
    finally:
        runtime.close()
    return 0


__all__ = ['count_roots', 'list_roots', 'root_bounds', 'genuine_cube_count', 'checker_record', 'ROOT_MAX', 'P_MAX']

if __name__ == '__main__':
    sys.exit(main(sys.argv[1:]))
