"""CPU oracle for the pseudocube sieve hot path.

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, and only as the checker.  The product package never imports it.

It restates, independently of ``psuedocubes_b200``, the reference's host arithmetic and batch
semantics (file:line refer to the reference project):

* ``primes``/``allowed``          pseudocube/tables.py:9-23 and pseudocube/oracle.py:7-11
* ``local3``/``icbrt``/``verify`` pseudocube/oracle.py:19-45, review/verify_cube.py:8-20
* ``Geometry``                    pseudocube/focus.py:97-121,189-210 (factors, coefficient-adjusted
                                  rings, CRT terms, halves, canonical pair, exact u interval, residual
                                  order of batch_experiment.py:84-86)
* ``OracleFocus.window``          pseudocube/gpu.py:94-114 + review/focus_window_cpu.cpp:4-25 (C code
                                  in sieve.c)
* ``batch``                       pseudocube/batch_experiment.py:27-57 (subtile geometry) and
                                  :104-167 (per-subtile scopes, digests, ordering) over the C masked
                                  matcher in sieve.c (:184-234)
* ``lease``                       pseudocube/optimized.py:26-90 (transcript over encoded scopes)
* ``encoded``/``digest``          pseudocube/accounting.py:17-32

Pinned against the reference's own golden lease replay
(results/continuation-2026-09-15/positive-lease-replay.json), the reference's enumerate_cpu on the
small complete sets, its focus_window_cpu.cpp and wide.c compiled into oracle/_ref, and its
known answers; see tests/test_oracle_pins.py.
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os
import subprocess
from concurrent.futures import ThreadPoolExecutor
from functools import lru_cache
from math import gcd, isqrt, prod
from pathlib import Path
from typing import Any

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / '_build' / 'libsieve_oracle.so'
REF_DIR = HERE / '_ref'

A619 = 701856356111039402
B619 = 693110504329192503
MASK64 = (1 << 64) - 1


# ---------------------------------------------------------------------------------------------
# exact host arithmetic

@lru_cache(maxsize=None)
def primes(p: int) -> tuple[int, ...]:
    return tuple(q for q in range(2, p + 1) if all(q % d for d in range(2, isqrt(q) + 1)))


@lru_cache(maxsize=None)
def allowed(q: int) -> tuple[int, ...]:
    if q == 9:
        return (1, 8)
    if q % 3 == 1:
        return tuple(sorted({a * a * a % q for a in range(1, q)}))
    return tuple(range(1, q))


def icbrt(n: int) -> int:
    lo, hi = 0, 1 << ((n.bit_length() + 2) // 3)
    while lo < hi:
        mid = (lo + hi + 1) // 2
        if mid ** 3 <= n:
            lo = mid
        else:
            hi = mid - 1
    return lo


def local3(n: int, p: int) -> bool:
    if n <= 0 or n % 9 not in (1, 8):
        return False
    return all(n % q and (q % 3 != 1 or pow(n, (q - 1) // 3, q) == 1) for q in primes(p))


def is_cube(n: int) -> bool:
    return n >= 0 and icbrt(n) ** 3 == n


def verify(n: int, p: int) -> dict[str, Any]:
    root = icbrt(n)
    failures = [q for q in primes(p) if n % q == 0 or (q % 3 == 1 and pow(n, (q - 1) // 3, q) != 1)]
    valid = n > 0 and n % 9 in (1, 8) and not failures and root ** 3 != n
    return dict(n=str(n), p=p, cube_root_floor=str(root), perfect_cube=root ** 3 == n,
                failing_primes=failures, valid_pseudocube=valid,
                claim='Candidate validity only; no minimality claim.')


def interoperable(value: Any) -> Any:
    if type(value) is int and abs(value) >= 1 << 53:
        return str(value)
    if isinstance(value, dict):
        return {str(k): interoperable(v) for k, v in value.items()}
    if isinstance(value, (list, tuple)):
        return [interoperable(v) for v in value]
    return value


def encoded(value: Any) -> bytes:
    return (json.dumps(interoperable(value), sort_keys=True, separators=(',', ':'),
                       allow_nan=False) + '\n').encode()


def digest(value: Any) -> str:
    return hashlib.sha256(encoded(value)).hexdigest()


# ---------------------------------------------------------------------------------------------
# geometry

class Geometry:
    """Focus rings, terms and residual filters of one (p, lo, hi, A, B)."""

    def __init__(self, p: int, lo: int, hi: int, A: int, B: int) -> None:
        if p % 3 != 1 or p not in primes(p) or not 0 <= lo < hi <= 3 * 10**27 or gcd(A, B) != 1:
            raise ValueError('invalid oracle geometry')
        self.p, self.lo, self.hi, self.A, self.B = p, lo, hi, A, B
        self.a_factors, self.b_factors = self._factors(A), self._factors(B)
        focus_set = set(self.a_factors) | set(self.b_factors)
        residuals = [q for q in [9, *primes(p)] if q != 3 and q not in focus_set]
        residuals.sort(key=lambda q: (q != 9 and q % 3 != 1, q))
        self.residuals = residuals
        self.filter_groups = [residuals[i:i + 4] for i in range(0, len(residuals), 4)]

    def _factors(self, n: int) -> list[int]:
        out = []
        for q in primes(self.p):
            if n % q:
                continue
            power = 1
            while n % q == 0:
                n //= q
                power *= q
            out.append(power)
        if n != 1:
            raise ValueError('focus prime above p')
        return out

    def rings(self, which: str) -> list[tuple[int, tuple[int, ...]]]:
        modulus, coefficient, factors = ((self.A, self.B, self.a_factors) if which == 'A'
                                         else (self.B, -self.A, self.b_factors))
        return [(q, tuple(sorted({a * pow(coefficient, -1, q) % q for a in allowed(q)})))
                for q in factors]

    def terms(self, which: str) -> list[list[int]]:
        M = self.A if which == 'A' else self.B
        return [[a * (M // q) * pow(M // q, -1, q) % M for a in res] for q, res in self.rings(which)]

    def canonical(self, n: int) -> tuple[int, int]:
        v = (-n * pow(self.A, -1, self.B)) % self.B if self.B > 1 else 0
        return (n + v * self.A) // self.B, v

    def u_interval(self, v: int) -> tuple[int, int]:
        return (self.lo + v * self.A) // self.B + 1, (self.hi + v * self.A) // self.B + 1

    def tile_ranges(self, first: int, end: int, width: int) -> list[tuple[int, int, int, int]]:
        if not 0 <= first < end <= self.B or width <= 0 or (end - first + width - 1) // width > 64:
            raise ValueError('invalid batch geometry')
        return [(v, min(v + width, end), self.u_interval(v)[0], self.u_interval(min(v + width, end) - 1)[1])
                for v in range(first, end, width)]

    def residual_arrays(self) -> tuple[np.ndarray, np.ndarray]:
        table = []
        for q in self.residuals:
            ring = [0] * q
            for a in allowed(q):
                ring[a] = 1
            table.extend(ring)
        return (np.array(self.residuals, dtype=np.uint32),
                np.array(table or [0], dtype=np.uint8))


# ---------------------------------------------------------------------------------------------
# the C restatement

_U64P = np.ctypeslib.ndpointer(dtype=np.uint64, flags='C_CONTIGUOUS')
_U32P = np.ctypeslib.ndpointer(dtype=np.uint32, flags='C_CONTIGUOUS')
_U8P = np.ctypeslib.ndpointer(dtype=np.uint8, flags='C_CONTIGUOUS')


def build() -> None:
    """Compile sieve.c (and, where the reference tree exists, its review tools)."""
    subprocess.run(['make', '-s', '-C', str(HERE)], check=True)


@lru_cache(maxsize=1)
def lib() -> ctypes.CDLL:
    if not LIB_PATH.exists():
        build()
    so = ctypes.CDLL(str(LIB_PATH))
    u64, u32 = ctypes.c_uint64, ctypes.c_uint32
    so.oc_partial.argtypes = [_U64P, _U32P, u32, u64, _U64P, u64]
    so.oc_sort_u64.argtypes = [_U64P, u64]
    so.oc_sort_u64.restype = None
    so.oc_window.argtypes = [_U64P, u64, _U64P, u64, u64, u64, u64, _U64P, u64, ctypes.POINTER(u64)]
    so.oc_wide.argtypes = [_U64P, _U64P, u64]
    so.oc_wide.restype = None
    so.oc_masked_batch.argtypes = [_U64P, u64, _U64P, u64, u64, u64, u64, u64, u64, u64,
                                   _U32P, u32, _U8P, u64, u64, u32, u64, _U64P, _U64P, ctypes.c_int]
    so.oc_plain_tile.argtypes = [_U64P, u64, _U64P, u64, u64, u64, u64, u64, u64, u64,
                                 _U32P, u32, _U8P, u64, _U64P, _U64P]
    so.oc_json_strings_u64.argtypes = [_U64P, u64, ctypes.c_char_p, u64]
    so.oc_json_strings_u64.restype = u64
    so.oc_cube_roots.argtypes = [u64, u64, u32, ctypes.c_void_p, u64, ctypes.POINTER(u64), ctypes.c_int]
    return so


def cube_roots(first: int, last: int, p: int, listed: bool = False, threads: int = 1) -> Any:
    """Roots a in [first, last] coprime to every prime <= p (review/cube_count.c:12-37): the
    count, or with ``listed`` the ascending roots as a uint32 array."""
    count = ctypes.c_uint64()
    if not listed:
        rc = lib().oc_cube_roots(first, last, p, None, 0, ctypes.byref(count), threads)
        if rc:
            raise ValueError(f'oracle cube roots rejected ({rc})')
        return count.value
    cap = last - first + 1 if 1 <= first <= last else 0
    out = np.zeros(max(1, cap), dtype=np.uint32)
    rc = lib().oc_cube_roots(first, last, p, out.ctypes.data, cap, ctypes.byref(count), 1)
    if rc:
        raise ValueError(f'oracle cube roots rejected ({rc})')
    return out[:count.value]


def wide(cases: np.ndarray) -> np.ndarray:
    cases = np.ascontiguousarray(cases, dtype=np.uint64).reshape(-1)
    out = np.zeros(len(cases) // 4 * 3, dtype=np.uint64)
    lib().oc_wide(cases, out, len(cases) // 4)
    return out.reshape(-1, 3)


def partial(rings: list[list[int]], M: int) -> np.ndarray:
    count = prod(len(t) for t in rings) if rings else 1
    terms = np.array([t for ring in rings for t in ring] or [0], dtype=np.uint64)
    sizes = np.array([len(t) for t in rings] or [1], dtype=np.uint32)
    out = np.zeros(count, dtype=np.uint64)
    if not rings:
        return out
    rc = lib().oc_partial(terms, sizes, len(rings), M, out, count)
    if rc:
        raise ValueError('oracle partial sums rejected')
    return out


def halves(terms: list[list[int]]) -> tuple[list[list[int]], list[list[int]]]:
    """Balanced two-way ring split (pseudocube/focus.py:81-87)."""
    best = min(range(1 << len(terms)), key=lambda mask: max(
        prod(len(t) for i, t in enumerate(terms) if mask & (1 << i)),
        prod(len(t) for i, t in enumerate(terms) if not mask & (1 << i))))
    return ([t for i, t in enumerate(terms) if best & (1 << i)],
            [t for i, t in enumerate(terms) if not best & (1 << i)])


@lru_cache(maxsize=1)
def reference_producer() -> ctypes.CDLL | None:
    """The reference's own window producer, review/focus_window_cpu.cpp compiled into
    oracle/_ref by the Makefile (None where it was not built)."""
    path = REF_DIR / 'focus_window.so'
    if not path.exists():
        return None
    so = ctypes.CDLL(str(path))
    u64 = ctypes.c_uint64
    so.focus_window.argtypes = [_U64P, u64, _U64P, u64, u64, u64, u64, u64, ctypes.c_void_p, u64, ctypes.POINTER(u64)]
    so.focus_window.restype = ctypes.c_int
    return so


class OracleFocus:
    """Sorted half sums C and D of one focus and the window query over them.  ``producer`` is
    'port' (the C restatement in sieve.c) or 'reference' (the reference's focus_window_cpu.cpp from
    oracle/_ref, one within-period call per period, then the same sort)."""

    producer = 'port'

    def __init__(self, geometry: Geometry, which: str) -> None:
        self.M = geometry.A if which == 'A' else geometry.B
        first, second = halves(geometry.terms(which))
        self.C = partial(first, self.M)
        lib().oc_sort_u64(self.C, len(self.C))
        self.D = partial(second, self.M)
        lib().oc_sort_u64(self.D, len(self.D))
        self.count = len(self.C) * len(self.D)

    def _reference_window(self, low: int, high: int, cap: int) -> np.ndarray:
        so = reference_producer()
        if so is None:
            raise RuntimeError('oracle/_ref/focus_window.so is not built')
        if high == low:
            return np.zeros(0, dtype=np.uint64)
        p0, p1 = low // self.M, (high - 1) // self.M
        if p1 - p0 + 1 > 4096:
            raise OverflowError('oracle window overflow')
        size = min(cap, 2 * self.count * (high - low) // self.M + 4096)
        out = np.zeros(max(1, size), dtype=np.uint64)
        written = 0
        count = ctypes.c_uint64()
        for period in range(p0, p1 + 1):
            base = period * self.M
            a, b = max(low, base) - base, min(high - base, self.M)
            while True:
                view = out[written:]
                rc = so.focus_window(self.C, len(self.C), self.D, len(self.D), self.M, a, b, base,
                                     view.ctypes.data, len(view), ctypes.byref(count))
                if rc != 1:
                    break
                if len(out) >= cap:
                    raise OverflowError('oracle window overflow')
                out = np.concatenate([out, np.zeros(min(cap, 4 * len(out)) - len(out), dtype=np.uint64)])
            if rc:
                raise ValueError('reference window producer rejected the window')
            written += count.value
        result = out[:written].copy()
        lib().oc_sort_u64(result, len(result))
        return result

    def window(self, low: int, high: int, cap: int = 10**6) -> np.ndarray:
        if not 0 <= low <= high < 1 << 64:
            raise ValueError('invalid window')
        if self.producer == 'reference':
            return self._reference_window(low, high, cap)
        size = min(cap, 2 * self.count * (high - low) // self.M + 4096)
        while True:
            out = np.zeros(max(1, size), dtype=np.uint64)
            count = ctypes.c_uint64()
            rc = lib().oc_window(self.C, len(self.C), self.D, len(self.D), self.M, low, high, out,
                                 len(out), ctypes.byref(count))
            if rc != 1 or size >= cap:
                break
            size = min(cap, 4 * size)
        if rc == 1 or count.value > cap:
            raise OverflowError('oracle window overflow')
        if rc:
            raise ValueError('oracle window rejected')
        return out[:count.value].copy()


def sorted_values(limbs: np.ndarray) -> list[int]:
    return sorted(int(a) | (int(b) << 64) for a, b in limbs.reshape(-1, 2))


def batch(geometry: Geometry, fa: OracleFocus, fb: OracleFocus, first: int, end: int,
          width: int = 100_000_000, output_cap: int = 8192, threads: int | None = None,
          verify_values: bool = True) -> dict[str, Any]:
    """One masked batch with the reference's result fields (timings omitted)."""
    g = geometry
    ranges = g.tile_ranges(first, end, width)
    us = fa.window(ranges[0][2], ranges[-1][3], cap=1 << 40)
    vs = fb.window(first, end, cap=1 << 40)
    ub = np.searchsorted(us, np.array([b for _, _, lo, hi in ranges for b in (lo, hi)], dtype=np.uint64)).reshape(-1, 2)
    vb = np.searchsorted(vs, np.array([b for lo, hi, _, _ in ranges for b in (lo, hi)], dtype=np.uint64)).reshape(-1, 2)
    bounds = [(int(a), int(b), int(c), int(d)) for (a, b), (c, d) in zip(ub, vb)]
    primes_arr, table = g.residual_arrays()
    ng = len(g.filter_groups)
    nt = len(ranges)
    counts = np.zeros(nt * (ng + 3), dtype=np.uint64)
    out = np.zeros(max(1, nt * 2 * output_cap), dtype=np.uint64)
    rc = lib().oc_masked_batch(us, len(us), vs, len(vs), g.A, g.B, g.lo & MASK64, g.lo >> 64,
                               g.hi & MASK64, g.hi >> 64, primes_arr, len(g.residuals), table,
                               first, width, nt, output_cap, counts, out, threads or os.cpu_count() or 1)
    if rc:
        raise RuntimeError(f'oracle batch failed ({rc})')
    pops = counts.reshape(nt, ng + 3)
    if np.any(pops[:, ng + 2]):
        raise ArithmeticError('unsigned underflow')
    if np.any(pops[:, ng + 1] > output_cap):
        raise OverflowError('oracle subtile output overflow')
    scopes, all_values = [], []
    for row, (lo_v, hi_v, _, _) in enumerate(ranges):
        number = int(pops[row, ng + 1])
        values = sorted_values(out[row * 2 * output_cap: row * 2 * output_cap + 2 * number])
        all_values.extend(values)
        scopes.append(dict(first=str(lo_v), end=str(hi_v), valid_focused_candidates=int(pops[row, 0]),
                           group_survivors=[int(n) for n in pops[row, 1:ng + 1]], local_survivors=number,
                           output_sha256=digest([str(n) for n in values])))
    if verify_values:
        bad = [n for n in all_values if not (g.lo < n <= g.hi and local3(n, g.p))]
        if bad:
            raise ArithmeticError(f'oracle emitted a non-survivor {bad[0]}')
    hits = [verify(n, g.p) for n in all_values if not is_cube(n)]
    return dict(focus_u=sum(b - a for a, b, _, _ in bounds), focus_v=len(vs),
                cartesian_opportunities=sum((b - a) * (d - c) for a, b, c, d in bounds),
                valid_focused_candidates=int(pops[:, 0].sum()),
                genuine_cubes=len(all_values) - len(hits), local_survivors=len(all_values),
                cube_checks=len(all_values), subtile_scopes=scopes, filter_groups=g.filter_groups,
                group_survivors=[int(n) for n in pops[:, 1:ng + 1].sum(axis=0)],
                all_values=[str(n) for n in all_values], cpu_confirmed_hits=hits)


BATCH_WIDTH = 100_000_000 * 64
LEASE_BATCHES = 256


def lease(geometry: Geometry, fa: OracleFocus, fb: OracleFocus, first: int, end: int,
          workers: int = 4, threads_per_batch: int = 2) -> dict[str, Any]:
    """Compact lease receipt fields (pseudocube/optimized.py:26-78), timings omitted."""
    starts = list(range(first, end, BATCH_WIDTH))

    def one(start: int) -> dict[str, Any]:
        return batch(geometry, fa, fb, start, min(start + BATCH_WIDTH, end), threads=threads_per_batch)

    with ThreadPoolExecutor(max_workers=workers) as pool:
        rows = list(pool.map(one, starts))
    transcript = hashlib.sha256()
    counts = dict.fromkeys(('focus_u', 'focus_v', 'cartesian_opportunities', 'valid_focused_candidates',
                            'genuine_cubes', 'local_survivors', 'cube_checks'), 0)
    groups = [0] * len(geometry.filter_groups)
    values: list[str] = []
    hits: list[dict[str, Any]] = []
    for row in rows:
        for k in counts:
            counts[k] += int(row[k])
        for i, n in enumerate(row['group_survivors']):
            groups[i] += n
        values.extend(row['all_values'])
        hits.extend(row['cpu_confirmed_hits'])
        transcript.update(encoded(row['subtile_scopes']))
    return dict(**counts, group_survivors=groups, filter_groups=geometry.filter_groups, all_values=values,
                cpu_confirmed_hits=hits, compute_batches=len(rows),
                subtiles_executed=sum(len(r['subtile_scopes']) for r in rows),
                transcript_sha256=transcript.hexdigest(), output_sha256=digest(values), batches=rows)


def plain_tile(geometry: Geometry, us: np.ndarray, vs: np.ndarray, output_cap: int = 8192) -> dict[str, Any]:
    """Plain per-tile matcher counters (pseudocube/gpu.py:129-182,199-234)."""
    g = geometry
    primes_arr, table = g.residual_arrays()
    ng = len(g.filter_groups)
    counts = np.zeros(ng + 3, dtype=np.uint64)
    out = np.zeros(max(1, 2 * output_cap), dtype=np.uint64)
    lib().oc_plain_tile(np.ascontiguousarray(us, dtype=np.uint64), len(us),
                        np.ascontiguousarray(vs, dtype=np.uint64), len(vs), g.A, g.B,
                        g.lo & MASK64, g.lo >> 64, g.hi & MASK64, g.hi >> 64, primes_arr,
                        len(g.residuals), table, output_cap, counts, out)
    number = int(counts[ng + 1])
    values = sorted_values(out[:2 * min(number, output_cap)])
    return dict(populations=[int(c) for c in counts], values=values)


def strings_digest_u64(values: np.ndarray) -> str:
    """digest([str(n) for n in values]) for long uint64 lists (values must already be in order)."""
    values = np.ascontiguousarray(values, dtype=np.uint64)
    cap = 24 * len(values) + 16
    buf = ctypes.create_string_buffer(cap)
    n = lib().oc_json_strings_u64(values, len(values), buf, cap)
    if n == 0:
        raise ValueError('json buffer too small')
    return hashlib.sha256(buf.raw[:n]).hexdigest()
