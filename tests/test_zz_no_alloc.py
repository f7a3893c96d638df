"""The plain matcher entry point that allocates no device memory, against the allocating one.

pc_run_plain_static serves callers that cannot call cudaMalloc (inside stream capture, under an
allocator that already owns the device, or where cudaMalloc's implicit synchronisation is not
acceptable).  Its scratch is a static device array shared by every call, so this test calls it
twice in a row on the same inputs: a second call must not see the first call's counters.  This
file is collected last so a failure here leaves every other test already run.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from psuedocubes_b200 import _native as N
from psuedocubes_b200.focus import Config, Tile
from psuedocubes_b200.gpu import MASK, GPUFocus, Matcher
from psuedocubes_b200.tables import allowed

pytestmark = pytest.mark.gpu


def filter_tables(config: Config) -> tuple[np.ndarray, np.ndarray]:
    order = config.filter_order()
    table = []
    for q in order:
        ring = [0] * q
        for a in allowed(q):
            ring[a] = 1
        table.extend(ring)
    return np.array(order, dtype=np.uint32), np.array(table, dtype=np.uint8)


def run_static(config: Config, us: np.ndarray, vs: np.ndarray, cap: int) -> tuple[list[int], list[int]]:
    primes, table = filter_tables(config)
    ng = (len(primes) + 3) // 4
    counts = np.zeros(ng + 3, dtype=np.uint64)
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


@pytest.mark.parametrize('case', ['p619-tile', 'p31-complete'])
def test_static_scratch_matches_allocating_entry_point(runtime, case):
    if case == 'p619-tile':
        from psuedocubes_b200.focus import A619, B619
        config = Config(619, 10**27, 3 * 10**27, A619, B619)
        tile = Tile(100_000_000, 200_000_000)
    else:
        config = Config(31, 0, 100000, 14 * 19, 9 * 13 * 31)
        tile = Tile(0, config.B)
    af, bf = (GPUFocus(runtime, f) for f in config.focuses())
    us = af.window(config.u_interval(tile.first)[0], config.u_interval(tile.end - 1)[1])
    vs = bf.window(tile.first, tile.end)
    cap = 1 << 16
    want = run_allocating(runtime, config, us, vs, cap)
    host_us, host_vs = us.get(), vs.get()
    for _ in range(2):                       # the shared array keeps the previous call's contents
        assert run_static(config, host_us, host_vs, cap) == want
    assert want[0][0] > 0                     # the tile has focused positions


def test_static_scratch_rejects_oversized_tiles(runtime):
    from psuedocubes_b200.focus import A619, B619
    config = Config(619, 10**27, 3 * 10**27, A619, B619)
    primes, table = filter_tables(config)
    big = np.arange(1 << 21, dtype=np.uint64)          # 16 MiB of u values alone
    counts = np.zeros(64, dtype=np.uint64)
    out = np.zeros(2, dtype=np.uint64)
    err = ctypes.create_string_buffer(256)
    code = N.lib().pc_run_plain_static(0, big, len(big), big[:4].copy(), 4, config.A, config.B, 0, 0, 0, 0, primes,
                                       len(primes), table, counts, out, 1, err, len(err))
    assert code == N.PC_INVALID
    assert b'16 MiB static scratch' in err.value
