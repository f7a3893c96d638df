"""The plain matcher entry point that allocates no device memory, against the allocating one.

pc_run_plain_static serves callers that cannot call cudaMalloc: a process whose own allocator
has already taken the device's memory, or code that cannot accept cudaMalloc's implicit device
synchronisation.  Its scratch is a static device array shared by every call, so the parity test
calls it twice in a row on the same inputs (a second call must not see the first call's
counters), then a truncated call and an empty call after a full one.  The refusal tests need no
device: every size is checked before the library touches one.  This file is collected last so a
failure here leaves every other test already run.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import golden
from psuedocubes_b200 import _native as N
from psuedocubes_b200.focus import A619, B619, Config, Tile
from psuedocubes_b200.gpu import MASK, GPUFocus, Matcher
from psuedocubes_b200.tables import allowed

P619 = Config(619, 10**27, 3 * 10**27, A619, B619)
P31 = Config(31, 0, 100000, 14 * 19, 9 * 13 * 31)


def filter_tables(config: Config) -> tuple[np.ndarray, np.ndarray]:
    order = config.filter_order()
    table = []
    for q in order:
        ring = [0] * q
        for a in allowed(q):
            ring[a] = 1
        table.extend(ring)
    return np.array(order, dtype=np.uint32), np.array(table, dtype=np.uint8)


def raw_static() -> ctypes._CFuncPtr:
    """The entry point with untyped pointer arguments, so a test can pass NULL."""
    fn = ctypes.CDLL(str(N.LIB_PATH)).pc_run_plain_static
    p, u64 = ctypes.c_void_p, ctypes.c_uint64
    fn.argtypes = [ctypes.c_int, p, u64, p, u64, u64, u64, u64, u64, u64, u64, p, ctypes.c_uint32, p, p, p, u64,
                   ctypes.c_char_p, ctypes.c_int]
    return fn


def run_static(config: Config, us: np.ndarray, vs: np.ndarray, cap: int) -> tuple[list[int], list[int]]:
    primes, table = filter_tables(config)
    ng = (len(primes) + 3) // 4
    counts = np.full(ng + 3, 7, dtype=np.uint64)        # the call must write every counter
    out = np.zeros(2 * max(1, cap), dtype=np.uint64)
    err = ctypes.create_string_buffer(256)
    code = N.lib().pc_run_plain_static(0, N.u64(us), len(us), N.u64(vs), len(vs), config.A, config.B,
                                       config.lo & MASK, config.lo >> 64, config.hi & MASK, config.hi >> 64,
                                       primes, len(primes), table, counts, out, cap, err, len(err))
    assert code == N.PC_OK, err.value.decode()
    n = int(counts[ng + 1])
    values = sorted(int(a) | (int(b) << 64) for a, b in out[:2 * min(n, cap)].reshape(-1, 2))
    return [int(c) for c in counts], values


def run_allocating(runtime, config: Config, us, vs, cap: int) -> tuple[list[int], list[int]]:
    m = Matcher(runtime, config)
    ng = len(m.filter_groups)
    counts = np.zeros(ng + 3, dtype=np.uint64)
    out = np.zeros(2 * max(1, cap), dtype=np.uint64)
    runtime.call(runtime.lib.pc_run_plain(runtime.ctx, m.filters.handle, us.handle, us.offset, us.size, vs.handle,
                                          vs.offset, vs.size, config.lo & MASK, config.lo >> 64, config.hi & MASK,
                                          config.hi >> 64, counts, out, cap, None))
    n = int(counts[ng + 1])
    values = sorted(int(a) | (int(b) << 64) for a, b in out[:2 * min(n, cap)].reshape(-1, 2))
    return [int(c) for c in counts], values


def tile_lists(runtime, config: Config, tile: Tile):
    af, bf = (GPUFocus(runtime, f) for f in config.focuses())
    us = af.window(config.u_interval(tile.first)[0], config.u_interval(tile.end - 1)[1])
    vs = bf.window(tile.first, tile.end)
    return us, vs


@pytest.mark.gpu
@pytest.mark.parametrize('case', ['p619-tile', 'p31-complete'])
def test_static_scratch_matches_allocating_entry_point(runtime, oracle, case):
    config, tile = (P619, Tile(100_000_000, 200_000_000)) if case == 'p619-tile' else (P31, Tile(0, P31.B))
    us, vs = tile_lists(runtime, config, tile)
    cap = 1 << 16
    want = run_allocating(runtime, config, us, vs, cap)
    host_us, host_vs = us.get(), vs.get()
    for _ in range(2):                       # the shared array keeps the previous call's contents
        assert run_static(config, host_us, host_vs, cap) == want
    assert want[0][0] > 0                     # the tile has focused positions
    if case == 'p31-complete':                # the reference's complete set for p = 31, x <= 10^5
        fixture = next(c for c in golden('small_sets.json') if c['p'] == 31)
        values = want[1]
        assert len(values) == fixture['count']
        assert oracle.digest([str(n) for n in values]) == fixture['values_sha256']


@pytest.mark.gpu
def test_static_scratch_truncates_and_clears_like_the_allocating_entry_point(runtime):
    us, vs = tile_lists(runtime, P31, Tile(0, P31.B))
    host_us, host_vs = us.get(), vs.get()
    full = run_static(P31, host_us, host_vs, 1 << 16)
    survivors = full[0][len(full[0]) - 2]
    cap = 16
    assert survivors > cap
    got = run_static(P31, host_us, host_vs, cap)
    want = run_allocating(runtime, P31, us, vs, cap)
    assert got[0] == want[0] == full[0]       # every counter, including the untruncated output count
    assert len(got[1]) == cap and set(got[1]) <= set(full[1])
    # an empty v list after a full call: the kernel is skipped, the counters still start at zero
    counts, values = run_static(P31, host_us, host_vs[:0], cap)
    assert counts == [0] * len(counts) and values == []
    counts, values = run_static(P31, host_us[:0], host_vs, cap)
    assert counts == [0] * len(counts) and values == []


def test_static_scratch_refuses_sizes_before_touching_a_device():
    """Sizes past the 16 MiB array, including ones whose byte counts would wrap in 64 bits, and
    NULL tables are refused on the host; no device is needed to see it."""
    fn = raw_static()
    primes, table = filter_tables(P619)
    ng = (len(primes) + 3) // 4
    us = np.arange(4, dtype=np.uint64)
    counts = np.zeros(ng + 3, dtype=np.uint64)
    out = np.zeros(2, dtype=np.uint64)
    ptr = lambda a: a.ctypes.data if a is not None else None

    def call(nu=4, nv=4, cap=1, p=primes, t=table, o=out, device=0):
        err = ctypes.create_string_buffer(256)
        code = fn(device, ptr(us), nu, ptr(us), nv, P619.A, P619.B, 0, 0, 0, 0, ptr(p), len(primes), ptr(t),
                  ptr(counts), ptr(o), cap, err, len(err))
        return code, err.value

    for kwargs in (dict(cap=1 << 62), dict(cap=(1 << 64) - 1), dict(cap=1 << 61), dict(nu=1 << 62),
                   dict(nv=(1 << 64) - 1), dict(nu=1 << 21 | 1), dict(cap=(1 << 20) + 1)):
        code, err = call(**kwargs)
        assert code == N.PC_INVALID, kwargs
        assert b'16 MiB static scratch' in err, kwargs
    for kwargs in (dict(p=None), dict(t=None), dict(o=None), dict(device=-1), dict(device=64)):
        code, _ = call(**kwargs)
        assert code == N.PC_INVALID, kwargs


@pytest.mark.gpu
def test_static_scratch_rejects_oversized_tiles(runtime):
    primes, table = filter_tables(P619)
    big = np.arange(1 << 21, dtype=np.uint64)          # 16 MiB of u values alone
    counts = np.zeros(64, dtype=np.uint64)
    out = np.zeros(2, dtype=np.uint64)
    err = ctypes.create_string_buffer(256)
    code = N.lib().pc_run_plain_static(0, big, len(big), big[:4].copy(), 4, P619.A, P619.B, 0, 0, 0, 0, primes,
                                       len(primes), table, counts, out, 1, err, len(err))
    assert code == N.PC_INVALID
    assert b'16 MiB static scratch' in err.value
