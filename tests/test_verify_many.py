"""The column-wise verifier (verify_many) against the standalone witness verifier verify() and the
local predicate local3, value by value: random values, perfect cubes, edge values, and real
survivors of the p=67 split from the oracle; the large-output paths of verify_values use it."""
from __future__ import annotations

import random

import numpy as np
import pytest

from psuedocubes_b200.batch_experiment import verify_values
from psuedocubes_b200.focus import Config
from psuedocubes_b200.predicate import icbrt, local3
from psuedocubes_b200.verify import VECTOR_MIN, icbrt_many, verify, verify_many

M64 = (1 << 64) - 1


def limbs(values):
    return (np.array([v & M64 for v in values], dtype=np.uint64), np.array([v >> 64 for v in values], dtype=np.uint64))


def test_rows_and_local_test_match_one_by_one():
    rng = random.Random(619003)
    values = [rng.getrandbits(rng.choice([12, 40, 64, 65, 90, 95])) for _ in range(6000)]
    values += [a ** 3 for a in range(1, 4000, 13)] + [a ** 3 + d for a in (2 ** 31 + 11, 2 ** 32 - 2) for d in (-1, 0, 1)]
    values += [0, 1, 8, 9, 10, (1 << 96) - 1]
    lo, hi = limbs(values)
    assert [int(a) for a in icbrt_many(lo, hi)] == [icbrt(v) for v in values]
    for p in (7, 67, 619):
        ok, cube, rows = verify_many(lo, hi, p, threads=3)
        assert [bool(x) for x in ok] == [local3(v, p) for v in values]
        assert [bool(x) for x in cube] == [icbrt(v) ** 3 == v for v in values]
        want = [verify(v, p) for v in values if icbrt(v) ** 3 != v]
        assert len(rows) == len(want) and list(rows) == want and rows[-1] == want[-1] and rows[:3] == want[:3]
    with pytest.raises(ValueError):
        verify_many(lo, hi, 11)                       # p must be prime and 1 mod 3
    with pytest.raises(ValueError):
        verify_many(np.zeros(1, np.uint64), np.array([1 << 32], np.uint64), 67)


def test_survivors_of_the_p67_split(oracle):
    """Survivors of a slice of the p=67 domain (A = 2523326, B = 2486169) from the oracle: every
    one passes, cubes are told apart, and the rows equal verify()'s."""
    g = oracle.Geometry(67, 1, 10**13, 2523326, 2486169)
    got = oracle.batch(g, oracle.OracleFocus(g, 'A'), oracle.OracleFocus(g, 'B'), 0, 600, width=600,
                       output_cap=1 << 22)
    values = [int(n) for n in got['all_values']]
    assert len(values) > VECTOR_MIN
    lo, hi = limbs(values)
    ok, cube, rows = verify_many(lo, hi, 67)
    assert ok.all() and rows.all_valid
    assert int(cube.sum()) == got['genuine_cubes']
    sample = random.Random(3).sample(range(len(rows)), 300)
    noncubes = [v for v in values if icbrt(v) ** 3 != v]
    assert [rows[i] for i in sample] == [verify(noncubes[i], 67) for i in sample]
    config = Config(67, 1, 10**13, 2523326, 2486169)
    hits = verify_values(config, values)                # the column-wise branch
    assert len(hits) == len(values) - got['genuine_cubes'] and hits[0] == verify(noncubes[0], 67)
    with pytest.raises(ArithmeticError):
        verify_values(config, values[:-1] + [values[-1] + 9])   # fails the local test mod 9 or a prime
    with pytest.raises(ArithmeticError):
        verify_values(config, values + [values[0]])             # duplicate
