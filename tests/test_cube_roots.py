"""Genuine-cube control: the roots a in [first, last] coprime to every prime <= p.

The oracle (a segmented byte sieve in oracle/sieve.c) is pinned to the reference's recorded
full-interval count (38,322,775 at p = 619, results/completion-2026-09-16/cube_count*.json) and to
the output of both reference checkers (review/cube_count.c, review/cube_count_independent.c) on
list and count cases (tests/golden/cube_roots.json, made by make_golden.py).  The device sieve
(pc_cube_roots) must give the same counts and the same ascending lists.
"""
from __future__ import annotations

import hashlib
import os

import numpy as np
import pytest

from conftest import golden
from psuedocubes_b200 import cubes
from psuedocubes_b200.predicate import icbrt, primes_upto

FIX = golden('cube_roots.json')


def _same_list(case: dict, roots: np.ndarray) -> None:
    text = [str(int(a)) for a in roots]
    assert len(text) == case['count']
    assert [int(a) for a in text[:16]] == case['head'] and [int(a) for a in text[-16:]] == case['tail']
    assert hashlib.sha256(','.join(text).encode()).hexdigest() == case['sha256']


def test_oracle_matches_the_reference_checkers(oracle):
    for case in FIX['listed']:
        _same_list(case, oracle.cube_roots(case['first'], case['last'], case['p'], listed=True))
    for case in FIX['counted']:
        assert oracle.cube_roots(case['first'], case['last'], case['p'], threads=os.cpu_count() or 1) == case['count']
    for row in FIX['recorded']:
        assert (row['first'], row['last'], row['p'], row['count']) == (1000000001, 1442249570, 619, 38322775)
        assert oracle.cube_roots(row['first'], row['last'], row['p'], threads=os.cpu_count() or 1) == row['count']
    with pytest.raises(ValueError):
        oracle.cube_roots(0, 5, 619)


def test_root_bounds_and_argument_checks():
    assert cubes.root_bounds(10**27, 3 * 10**27) == (1000000001, 1442249570)
    assert cubes.root_bounds(7, 8) == (2, 2)                 # hi = 2^3 is inside (lo, hi]
    assert cubes.root_bounds(8, 26) is None                  # lo = 2^3 is outside
    assert cubes.root_bounds(0, 0) is None and cubes.root_bounds(5, 5) is None
    assert cubes.root_bounds(0, 1) == (1, 1)
    for first, last, p in ((0, 5, 619), (5, 4, 619), (1, 2**32, 619), (1, 5, 1), (1, 5, 2001)):
        with pytest.raises(ValueError):
            cubes._check(first, last, p)
    assert cubes.main(['1', '2']) == 2                       # usage errors exit 2 before any device use
    assert cubes.main(['5', '4', '619']) == 2
    assert cubes.main(['1', '200000', '619', '--list']) == 2


@pytest.mark.gpu
def test_device_counts_and_lists_match_the_reference(runtime):
    for case in FIX['listed']:
        roots = cubes.list_roots(runtime, case['first'], case['last'], case['p'])
        assert roots.dtype == np.uint32 and np.all(np.diff(roots.astype(np.int64)) > 0)
        _same_list(case, roots)
        assert cubes.count_roots(runtime, case['first'], case['last'], case['p']) == case['count']
    for case in FIX['counted']:
        assert cubes.count_roots(runtime, case['first'], case['last'], case['p']) == case['count'], case
    for row in FIX['recorded']:
        record = cubes.checker_record(runtime, row['first'], row['last'], row['p'])
        assert record['count'] == str(row['count']) and record['root_first'] == str(row['first'])
        assert record['root_last'] == str(row['last']) and record['p'] == row['p']


@pytest.mark.gpu
def test_device_list_overflow_and_invalid_bounds(runtime):
    from psuedocubes_b200 import _native as N
    import ctypes
    with pytest.raises(OverflowError):
        cubes.list_roots(runtime, 1, 100000, 619, cap=100)
    count = ctypes.c_uint64()
    out = np.zeros(16, dtype=np.uint32)
    assert runtime.lib.pc_cube_roots(runtime.ctx, 1, 100000, 619, out.ctypes.data, 16, ctypes.byref(count), None) == N.PC_OVERFLOW
    assert count.value == 9479
    for first, last, p in ((0, 5, 619), (5, 4, 619), (1, 2**32, 619), (1, 5, 1), (1, 5, 2001)):
        assert runtime.lib.pc_cube_roots(runtime.ctx, first, last, p, None, 0, ctypes.byref(count), None) == N.PC_INVALID
    assert cubes.list_roots(runtime, 8, 9, 2).tolist() == [9] and cubes.list_roots(runtime, 2, 2, 2).size == 0
    ends = cubes.list_roots(runtime, 2**32 - 40, 2**32 - 1, 7)
    assert ends.tolist() == [a for a in range(2**32 - 40, 2**32) if all(a % q for q in (2, 3, 5, 7))]


@pytest.mark.gpu
def test_genuine_cube_count_matches_an_independent_count(runtime):
    for p, lo, hi in ((619, 10**20, 10**20 + 10**18), (547, 10**27, 10**27 + 10**24), (31, 0, 10**12), (619, 26, 27)):
        ps = primes_upto(p)
        want = sum(1 for a in range(icbrt(lo) + 1, icbrt(hi) + 1) if all(a % q for q in ps))
        assert cubes.genuine_cube_count(runtime, p, lo, hi) == want
