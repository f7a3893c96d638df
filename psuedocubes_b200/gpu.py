"""Device runtime, focus windows and the plain per-tile matcher over libpcube.

Mirrors the call surface of pseudocube/gpu.py:38-252 (Runtime, GPUFocus, launch_plan, Matcher)
with CuPy/NVRTC replaced by the precompiled sm_100a library behind a ctypes C ABI.  There is no
CPU path: every method raises if the library or the GPU is unavailable.
"""
from __future__ import annotations

import ctypes
import time
from typing import Any

import numpy as np

from . import _native as N
from .focus import Config, Focus, Tile
from .predicate import is_perfect_cube, local3
from .tables import allowed

MASK = (1 << 64) - 1


def device_count() -> int:
    return N.device_count()


class Runtime:
    """One device context: stream, memory cap, deadline (pseudocube/gpu.py:38-52)."""

    def __init__(self, deadline: float, memory_cap: int, memory_fraction: float = 0.5, device: int = 0) -> None:
        self.deadline = deadline
        self.lib = N.lib()
        handle = ctypes.c_void_p()
        code = self.lib.pc_init(device, int(memory_cap), float(memory_fraction), ctypes.byref(handle))
        if code == N.PC_NOMEM:
            raise MemoryError('no permitted device memory')
        N.raise_for(code, None, 'cannot open the CUDA device')
        self.ctx = handle
        self.compiles: list[dict[str, Any]] = [N.library_record()]
        self.peak_device = 0
        sm, major, minor = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        name = ctypes.create_string_buffer(256)
        self.lib.pc_device_info(self.ctx, ctypes.byref(sm), ctypes.byref(major), ctypes.byref(minor), name, 256)
        self.sm_count, self.capability, self.device_name = sm.value, (major.value, minor.value), name.value.decode()

    @property
    def cap(self) -> int:
        return self.memory()[2]

    def memory(self) -> tuple[int, int, int]:
        in_use, peak, cap = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        self.lib.pc_mem_info(self.ctx, ctypes.byref(in_use), ctypes.byref(peak), ctypes.byref(cap))
        return in_use.value, peak.value, cap.value

    def copies(self) -> tuple[int, int]:
        """(host-to-device, device-to-host) bytes the library has copied on this context so far."""
        h2d, d2h = ctypes.c_uint64(), ctypes.c_uint64()
        self.call(self.lib.pc_copy_info(self.ctx, ctypes.byref(h2d), ctypes.byref(d2h)))
        return h2d.value, d2h.value

    def check(self) -> None:
        if time.monotonic() >= self.deadline - 3:
            raise TimeoutError('BUDGET_EXHAUSTED')
        in_use, peak, cap = self.memory()
        self.peak_device = max(self.peak_device, peak)
        if self.peak_device > cap:
            raise MemoryError('device memory cap exceeded')

    def call(self, code: int, what: str = '') -> None:
        N.raise_for(code, self.ctx, what)

    def synchronize(self) -> None:
        self.call(self.lib.pc_sync(self.ctx))

    def close(self) -> None:
        if getattr(self, 'ctx', None):
            self.lib.pc_free(self.ctx)
            self.ctx = None

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass


class DeviceArray:
    """A sorted uint64 array resident on the device (slices share the allocation)."""

    def __init__(self, runtime: Runtime, handle: ctypes.c_void_p, offset: int = 0, size: int | None = None,
                 owner: 'DeviceArray | None' = None) -> None:
        self.runtime, self.handle, self.offset = runtime, handle, offset
        if size is None:
            n = ctypes.c_uint64()
            runtime.lib.pc_buf_size(handle, ctypes.byref(n))
            size = n.value
        self.size = size
        self._owner = owner

    @classmethod
    def from_host(cls, runtime: Runtime, values: Any) -> 'DeviceArray':
        data = N.u64(values)
        handle = ctypes.c_void_p()
        runtime.call(runtime.lib.pc_buf_upload(runtime.ctx, data, len(data), ctypes.byref(handle)))
        return cls(runtime, handle)

    def __len__(self) -> int:
        return self.size

    def __getitem__(self, key: slice) -> 'DeviceArray':
        if not isinstance(key, slice) or key.step not in (None, 1):
            raise TypeError('device arrays support contiguous slices only')
        start, stop, _ = key.indices(self.size)
        stop = max(start, stop)
        return DeviceArray(self.runtime, self.handle, self.offset + start, stop - start, self._owner or self)

    def get(self) -> np.ndarray:
        out = np.zeros(self.size, dtype=np.uint64)
        if self.size:
            self.runtime.call(self.runtime.lib.pc_buf_download(self.runtime.ctx, self.handle, self.offset,
                                                               self.size, out))
        return out

    def searchsorted(self, queries: Any) -> np.ndarray:
        """Left insertion points of sorted-order queries, relative to this (sorted) slice."""
        q = N.u64(queries)
        out = np.zeros(len(q), dtype=np.uint64)
        if len(q):
            self.runtime.call(self.runtime.lib.pc_buf_searchsorted(self.runtime.ctx, self.handle, q, len(q), out))
            # the whole allocation is sorted, so a slice's answer is the clamped global answer
            out = np.clip(out.astype(np.int64) - self.offset, 0, self.size).astype(np.uint64)
        return out

    def __del__(self) -> None:
        if self._owner is None and getattr(self, 'handle', None) and self.runtime.ctx:
            try:
                self.runtime.lib.pc_buf_free(self.runtime.ctx, self.handle)
            except Exception:
                pass
            self.handle = None


class GPUFocus:
    """Device-resident wheel tables of one focus and its sorted window query
    (pseudocube/gpu.py:70-114).  The reference's sorted/unsorted half-sum arrays C and D are
    replaced by a wheel W1 over a sub-modulus and bitset rows of the largest rings."""

    def __init__(self, runtime: Runtime, focus: Focus, table_budget: int = 0) -> None:
        self.runtime, self.focus = runtime, focus
        qs = np.array([q for q, _ in focus.rings] or [1], dtype=np.uint32)
        counts = np.array([len(r) for _, r in focus.rings] or [1], dtype=np.uint32)
        residues = np.array([a for _, r in focus.rings for a in r] or [0], dtype=np.uint32)
        handle = ctypes.c_void_p()
        runtime.check()
        runtime.call(runtime.lib.pc_focus_create(runtime.ctx, focus.modulus, len(focus.rings), qs, counts,
                                                 residues, table_budget, ctypes.byref(handle)))
        self.handle = handle
        info = np.zeros(8, dtype=np.uint64)
        runtime.lib.pc_focus_info(handle, info)
        self.modulus, self.wheel_modulus, self.wheel_size = int(info[0]), int(info[1]), int(info[2])
        self.bitset_rings, self.table_bytes = int(info[3]), int(info[4])
        self.count = int(info[5]) | (int(info[6]) << 64)
        if self.count != focus.count:
            raise ArithmeticError('device focus count disagrees with the ring counts')
        self.half_sizes = [self.wheel_size, self.bitset_rings]
        self.build_ms = int(info[7])
        runtime.check()

    def window(self, low: int, high: int, cap: int = 1000000) -> DeviceArray:
        if not 0 <= low <= high < 1 << 64:
            raise ValueError('invalid bounded focus window')
        handle = ctypes.c_void_p()
        count = ctypes.c_uint64()
        self.runtime.check()
        self.runtime.call(self.runtime.lib.pc_focus_window(self.runtime.ctx, self.handle, low, high, cap,
                                                           ctypes.byref(handle), ctypes.byref(count)))
        return DeviceArray(self.runtime, handle, 0, count.value)

    def __del__(self) -> None:
        if getattr(self, 'handle', None) and self.runtime.ctx:
            try:
                self.runtime.lib.pc_focus_free(self.runtime.ctx, self.handle)
            except Exception:
                pass
            self.handle = None


class Filters:
    """Residual filter tables of one config on the device, in the reference's filter order."""

    def __init__(self, runtime: Runtime, config: Config, table: Any = None) -> None:
        """``table`` replaces the residue table uploaded to the device: one byte per residue r of
        each filter q (1 = allowed), concatenated in filter order.  The default is the allowed
        residues of each filter; another table is how a qualification run checks that the host
        re-verification catches wrong device tables (the reference mutates its device table for
        that, tools/gpu_worker.py:96-103 of its release archive)."""
        self.runtime, self.config = runtime, config
        order = config.filter_order()
        if not order:
            raise ValueError('bitset experiment requires at least one residual filter')
        self.order = order
        self.filter_groups = [order[i:i + 4] for i in range(0, len(order), 4)]
        self.ng = len(self.filter_groups)
        if table is None:
            table = []
            for q in order:
                ring = [0] * q
                for a in allowed(q):
                    ring[a] = 1
                table.extend(ring)
        elif len(table) != sum(order):
            raise ValueError('residue table must hold one byte per residue of every filter')
        handle = ctypes.c_void_p()
        runtime.call(runtime.lib.pc_filters_create(runtime.ctx, config.A, config.B,
                                                   np.array(order, dtype=np.uint32), len(order),
                                                   np.array(table, dtype=np.uint8), ctypes.byref(handle)))
        self.handle = handle

    def __del__(self) -> None:
        if getattr(self, 'handle', None) and self.runtime.ctx:
            try:
                self.runtime.lib.pc_filters_free(self.runtime.ctx, self.handle)
            except Exception:
                pass
            self.handle = None


def launch_plan(nu: int, nv: int, sm_count: int, layout: str, blocks_per_sm: int = 2) -> tuple[int, int]:
    """(blocks, warps per v row) of the reference's row-striped layout (pseudocube/gpu.py:117-126);
    kept for the plain matcher's launch description and its argument checks."""
    if layout not in ('serial', 'warp') or type(blocks_per_sm) is not int or blocks_per_sm not in (1, 2, 4):
        raise ValueError('invalid matching layout')
    if min(nu, nv) < 0 or sm_count < 1:
        raise ValueError('invalid launch dimensions')
    if not nu or not nv:
        return 0, 1
    if layout == 'serial':
        return (nv + 255) // 256, 1
    stripes = min((nu + 31) // 32, max(1, (sm_count * blocks_per_sm * 8 + nv - 1) // nv))
    return (nv * stripes + 7) // 8, stripes


def limbs_to_values(limbs: np.ndarray) -> list[int]:
    pairs = limbs.reshape(-1, 2)
    return [int(a) | (int(b) << 64) for a, b in pairs]


class Matcher:
    """Plain per-tile matcher: every residual filter tested per position (pseudocube/gpu.py:185-252)."""

    def __init__(self, runtime: Runtime, config: Config, variant: str = 'byte', layout: str = 'warp',
                 blocks_per_sm: int = 2) -> None:
        if variant not in ('byte', 'packed', 'constant'):
            raise ValueError('unknown lookup variant')
        if layout not in ('serial', 'warp'):
            raise ValueError('unknown matching layout')
        launch_plan(0, 0, max(1, runtime.sm_count), layout, blocks_per_sm)
        self.runtime, self.config, self.variant = runtime, config, variant
        self.layout, self.blocks_per_sm = layout, blocks_per_sm
        self.sm_count = runtime.sm_count
        self.filters = Filters(runtime, config)
        self.filter_groups = self.filters.filter_groups

    def arrays(self, us: DeviceArray, vs: DeviceArray, cap: int = 8192) -> dict[str, Any]:
        started = time.perf_counter()
        ng = len(self.filter_groups)
        if us.size * vs.size > 50_000_000:
            raise OverflowError('bounded pair-opportunity limit exceeded')
        if cap < 0:
            raise ValueError('negative output capacity')
        blocks, stripes = launch_plan(us.size, vs.size, self.sm_count, self.layout, self.blocks_per_sm)
        counts = np.zeros(ng + 3, dtype=np.uint64)
        out = np.zeros(max(2, 2 * cap), dtype=np.uint64)
        stats = N.Stats()
        c = self.config
        self.runtime.check()
        self.runtime.call(self.runtime.lib.pc_run_plain(
            self.runtime.ctx, self.filters.handle, us.handle, us.offset, us.size, vs.handle, vs.offset, vs.size,
            c.lo & MASK, c.lo >> 64, c.hi & MASK, c.hi >> 64, counts, out, cap, ctypes.byref(stats)))
        self.runtime.check()
        transfer = time.perf_counter()
        populations = [int(x) for x in counts]
        number = populations[ng + 1]
        if populations[ng + 2]:
            raise ArithmeticError('unsigned underflow flagged')
        if number > cap:
            raise OverflowError('output overflow; attempt cannot commit')
        values = sorted(limbs_to_values(out[:2 * number]))
        transfer = time.perf_counter() - transfer
        verification = time.perf_counter()
        if len(values) != len(set(values)):
            raise ArithmeticError('duplicate canonical output')
        if any(not c.lo < n <= c.hi or not local3(n, c.p) for n in values):
            raise ArithmeticError('GPU/CPU disagreement: attempt quarantined')
        cube_flags = [is_perfect_cube(n) for n in values]
        cubes = [n for n, flag in zip(values, cube_flags) if flag]
        hits = [n for n, flag in zip(values, cube_flags) if not flag]
        verification = time.perf_counter() - verification
        return dict(status='PASS', host_verified=True, variant=self.variant, focus_u=us.size, focus_v=vs.size,
                    layout=self.layout, blocks_per_sm=self.blocks_per_sm, warps_per_row=stripes,
                    launch_blocks=blocks, threads_per_block=256, launched_warps=blocks * 8,
                    cartesian_opportunities=us.size * vs.size, pairs_visited=populations[0],
                    valid_focused_candidates=populations[0], wide_constructions=populations[0],
                    filter_groups=self.filter_groups, group_survivors=populations[1:ng + 1], local_survivors=number,
                    cube_checks=number, genuine_cubes=len(cubes), noncube_reports=len(hits),
                    cpu_confirmed_hits=list(map(str, hits)), cpu_rejected_reports=0,
                    all_values=list(map(str, values)), kernel_seconds=stats.kernel_ms / 1000,
                    transfer_seconds=transfer, verification_seconds=verification,
                    end_to_end_seconds=time.perf_counter() - started)

    def coordinates(self, us: list[int], vs: list[int], cap: int = 8192) -> dict[str, Any]:
        started = time.perf_counter()
        u = DeviceArray.from_host(self.runtime, np.array(sorted(us), dtype=np.uint64))
        v = DeviceArray.from_host(self.runtime, np.array(vs, dtype=np.uint64))
        transfer = time.perf_counter() - started
        result = self.arrays(u, v, cap)
        result['input_transfer_seconds'] = transfer
        result['end_to_end_seconds'] = time.perf_counter() - started
        return result

    def tile(self, tile: Tile, af: GPUFocus, bf: GPUFocus, cap: int = 1000000, output_cap: int = 8192) -> dict[str, Any]:
        tile.validate(self.config)
        started = time.perf_counter()
        lower = self.config.u_interval(tile.first)[0]
        upper = self.config.u_interval(tile.end - 1)[1]
        us = af.window(lower, upper, cap)
        vs = bf.window(tile.first, tile.end, cap)
        prep = time.perf_counter() - started
        result = self.arrays(us, vs, output_cap)
        result['focus_enumeration_seconds'] = prep
        result['tile'] = tile.manifest(self.config)
        result['end_to_end_seconds'] = time.perf_counter() - started
        return result
