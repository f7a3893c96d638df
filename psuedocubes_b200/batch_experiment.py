"""Batched engines: one fused launch per batch of up to 64 subtiles.

Mirrors pseudocube/batch_experiment.py:16-263 (Prepared, tile_ranges, prepare_arrays, prepare,
CachedMatcher, FusedMatcher, MaskedMatcher, compare).  FusedMatcher and MaskedMatcher both call
the sm_100a fused kernel; they differ only in how many residual filters are intersected as
bitsets before exact 128-bit arithmetic takes over (the minimum the populations need, versus the
tuned tier).  Results, populations and subtile digests are identical by construction.
"""
from __future__ import annotations

import ctypes
import time
from collections.abc import Sequence
from dataclasses import dataclass
from typing import Any

import numpy as np

from . import _native as N
from .accounting import EMPTY_DIGEST, digest, scope_list
from .focus import Config, Tile
from .gpu import MASK, DeviceArray, Filters, GPUFocus, Matcher, Runtime, launch_plan
from .predicate import is_perfect_cube, local3
from .verify import MATERIALISE_MAX, VECTOR_MIN, verify, verify_many


@dataclass
class Prepared:
    first: int
    end: int
    width: int
    us: Any
    vs: Any
    bounds: list[tuple[int, int, int, int]]
    prep_seconds: float


def tile_ranges(config: Config, first: int, end: int, width: int) -> list[tuple[int, int, int, int]]:
    """Subtile v ranges with their inclusive u envelopes (pseudocube/batch_experiment.py:27-32)."""
    Tile(first, end).validate(config)
    if width <= 0 or (end - first + width - 1) // width > 64:
        raise ValueError('experiment allows at most 64 bounded subtiles')
    rows = []
    for v in range(first, end, width):
        stop = min(v + width, end)
        rows.append((v, stop, config.u_interval(v)[0], config.u_interval(stop - 1)[1]))
    return rows


def prepare_arrays(runtime: Runtime, config: Config, first: int, end: int, width: int,
                   us: DeviceArray, vs: DeviceArray, started: float) -> Prepared:
    ranges = tile_ranges(config, first, end, width)
    ub = us.searchsorted([b for _, _, lo, hi in ranges for b in (lo, hi)]).reshape(-1, 2)
    vb = vs.searchsorted([b for lo, hi, _, _ in ranges for b in (lo, hi)]).reshape(-1, 2)
    bounds = [(int(a), int(b), int(c), int(d)) for (a, b), (c, d) in zip(ub, vb)]
    for a, b, c, d in bounds:
        if (b - a) * (d - c) > 50_000_000:
            raise OverflowError('per-subtile candidate opportunity limit exceeded')
    runtime.check()
    return Prepared(first, end, width, us, vs, bounds, time.perf_counter() - started)


def prepare(runtime: Runtime, config: Config, af: GPUFocus, bf: GPUFocus, first: int, end: int,
            width: int = 100000000) -> Prepared:
    started = time.perf_counter()
    ranges = tile_ranges(config, first, end, width)
    us = af.window(ranges[0][2], ranges[-1][3])
    vs = bf.window(first, end)
    return prepare_arrays(runtime, config, first, end, width, us, vs, started)


class CachedMatcher(Matcher):
    """Plain matcher over the subtile slices of a prepared batch."""
    prepared: Prepared | None = None

    def tile(self, tile: Tile, af: GPUFocus, bf: GPUFocus, cap: int = 1000000, output_cap: int = 8192) -> dict[str, Any]:
        started = time.perf_counter()
        batch = self.prepared
        if batch is None or not batch.first <= tile.first < tile.end <= batch.end:
            raise ValueError('tile outside prepared batch')
        index, remainder = divmod(tile.first - batch.first, batch.width)
        if remainder or tile.end != min(tile.first + batch.width, batch.end):
            raise ValueError('unexpected prepared subtile geometry')
        a, b, c, d = batch.bounds[index]
        result = self.arrays(batch.us[a:b], batch.vs[c:d], output_cap)
        result['focus_enumeration_seconds'] = 0.0
        result['tile'] = tile.manifest(self.config)
        result['end_to_end_seconds'] = time.perf_counter() - started
        return result


def split_outputs(records: np.ndarray, ntiles: int) -> list[list[int]]:
    """Device output records (x limb 0, x limb 1 | subtile << 32) grouped by subtile, each sorted."""
    per: list[list[int]] = [[] for _ in range(ntiles)]
    if len(records):
        lo = records[:, 0]
        hi = records[:, 1] & np.uint64(0xFFFFFFFF)
        tile = (records[:, 1] >> np.uint64(32)).astype(np.int64)
        for t, a, b in zip(tile.tolist(), lo.tolist(), hi.tolist()):
            per[t].append(a | (b << 64))
        for t in set(tile.tolist()):
            per[t].sort()
    return per


def verify_values(config: Config, values: list[int]) -> Sequence[dict[str, Any]]:
    """Host re-check of every emitted value (pseudocube/batch_experiment.py:138-144).  Many values
    are checked column-wise on all host cores (verify_many: the same predicates, the same rows)."""
    if len(values) != len(set(values)):
        raise ArithmeticError('duplicate canonical output')
    if len(values) >= VECTOR_MIN and config.hi < 1 << 96:
        if any(not config.lo < n <= config.hi for n in (min(values), max(values))):
            raise ArithmeticError('GPU/CPU disagreement')
        lo = np.fromiter((n & MASK for n in values), dtype=np.uint64, count=len(values))
        hi = np.fromiter((n >> 64 for n in values), dtype=np.uint64, count=len(values))
        ok, _, hits = verify_many(lo, hi, config.p)
        if not ok.all():
            raise ArithmeticError('GPU/CPU disagreement')
        if not hits.all_valid:
            raise ArithmeticError('independent witness verification failed')
        return list(hits) if len(hits) <= MATERIALISE_MAX else hits
    if any(not config.lo < n <= config.hi or not local3(n, config.p) for n in values):
        raise ArithmeticError('GPU/CPU disagreement')
    hits = [verify(n, config.p) for n in values if not is_perfect_cube(n)]
    if any(not row['valid_pseudocube'] for row in hits):
        raise ArithmeticError('independent witness verification failed')
    return hits


def batch_result(config: Config, ranges: list[tuple[int, int, int, int]], pops: np.ndarray,
                 per_tile: list[list[int]], geometry: list[tuple[int, int]], filter_groups: list[list[int]],
                 output_cap: int) -> dict[str, Any]:
    """Result fields of one batch from its subtile counters (batch_experiment.py:122-167)."""
    ng = len(filter_groups)
    if np.any(pops[:, ng + 2]):
        raise ArithmeticError('unsigned underflow')
    if np.any(pops[:, ng + 1] > output_cap):
        raise OverflowError('fused tile output overflow; no truncated coverage')
    emitted = pops[:, ng + 1].tolist()
    all_values: list[int] = []
    digests = []
    for row, (first, end, _, _) in enumerate(ranges):
        values = per_tile[row]
        if len(values) != emitted[row]:
            raise ArithmeticError('device output count disagrees with its records')
        if values:
            if any(not first <= config.canonical(n)[1] < end for n in values):
                raise ArithmeticError('output assigned to wrong subtile')
            all_values.extend(values)
            digests.append(digest([str(n) for n in values]))
        else:
            digests.append(EMPTY_DIGEST)
    scopes = scope_list([r[0] for r in ranges], [r[1] for r in ranges], pops[:, 0].tolist(),
                        pops[:, 1:ng + 1].tolist(), emitted, digests,
                        below_2_53=int(pops[:, :ng + 2].max(initial=0)) < 1 << 53)
    hits = verify_values(config, all_values)
    groups = [int(n) for n in pops[:, 1:ng + 1].sum(axis=0)] if len(ranges) else [0] * ng
    return dict(status='PASS', host_verified=True, focus_u=sum(u for u, _ in geometry),
                focus_v=sum(v for _, v in geometry), cartesian_opportunities=sum(u * v for u, v in geometry),
                valid_focused_candidates=int(pops[:, 0].sum()), genuine_cubes=len(all_values) - len(hits),
                local_survivors=len(all_values), cube_checks=len(all_values), subtile_scopes=scopes,
                filter_groups=filter_groups, group_survivors=groups, all_values=[str(n) for n in all_values],
                cpu_confirmed_hits=hits, overflow_splits=[])


class FusedMatcher:
    """One fused launch per batch with per-subtile counters and outputs
    (pseudocube/batch_experiment.py:79-167); the minimal bitset tier."""
    bitset_filters = 4

    def __init__(self, runtime: Runtime, config: Config, tuning: dict[str, int] | None = None) -> None:
        self.runtime, self.config = runtime, config
        self.filters = Filters(runtime, config)
        self.filter_groups = self.filters.filter_groups
        self.sm_count = runtime.sm_count
        self.tuning = N.Tuning()
        settings = dict(bitset_filters=min(self.bitset_filters, len(self.filters.order)))
        settings.update(tuning or {})
        for key, value in settings.items():
            setattr(self.tuning, key, int(value))
        self.last_stats: dict[str, Any] = {}

    def run(self, batch: Prepared, output_cap: int = 8192) -> dict[str, Any]:
        started = time.perf_counter()
        ranges = tile_ranges(self.config, batch.first, batch.end, batch.width)
        if len(ranges) != len(batch.bounds) or not 0 < output_cap <= 8192:
            raise ValueError('invalid prepared geometry or output capacity')
        ng = len(self.filter_groups)
        nt = len(ranges)
        counts = np.zeros(nt * (ng + 3), dtype=np.uint64)
        geometry = np.zeros(2 * nt, dtype=np.uint64)
        capacity = nt * output_cap
        records = np.zeros(2 * capacity, dtype=np.uint64)
        n_out = ctypes.c_uint64()
        stats = N.Stats()
        c = self.config
        us, vs = batch.us, batch.vs
        self.runtime.check()
        code = self.runtime.lib.pc_run_batch(
            self.runtime.ctx, self.filters.handle, ctypes.byref(self.tuning), us.handle, us.offset, us.size,
            vs.handle, vs.offset, vs.size, c.lo & MASK, c.lo >> 64, c.hi & MASK, c.hi >> 64,
            batch.first, batch.width, nt, batch.end, counts, geometry, records, capacity, ctypes.byref(n_out),
            ctypes.byref(stats))
        if code == N.PC_OVERFLOW:
            raise OverflowError('fused tile output overflow; no truncated coverage')
        self.runtime.call(code)
        self.runtime.check()
        self.last_stats = stats.as_dict()
        transfer_started = time.perf_counter()
        pops = counts.reshape(nt, ng + 3)
        per_tile = split_outputs(records[:2 * n_out.value].reshape(-1, 2), nt)
        transfer_seconds = time.perf_counter() - transfer_started
        geo = [(b - a, d - c_) for a, b, c_, d in batch.bounds]
        device_geo = [(int(geometry[2 * i]), int(geometry[2 * i + 1])) for i in range(nt)]
        if device_geo != geo:
            raise ArithmeticError('device subtile geometry disagrees with the prepared bounds')
        verification_started = time.perf_counter()
        result = batch_result(c, ranges, pops, per_tile, geo, self.filter_groups, output_cap)
        result.update(kernel_seconds=stats.kernel_ms / 1000, transfer_seconds=transfer_seconds,
                      verification_seconds=time.perf_counter() - verification_started,
                      focus_enumeration_seconds=batch.prep_seconds,
                      elapsed_seconds=time.perf_counter() - started + batch.prep_seconds,
                      kernel_registers=None, kernel_local_bytes=None,
                      claim='Isolated validation only; no production coverage.', matching_layout='fused-batch')
        return result


class MaskedMatcher(FusedMatcher):
    """Residue bitsets of the first residual filters intersected before any wide construction
    (pseudocube/batch_experiment.py:170-254); the production engine."""
    bitset_filters = 7
    lease_output_records = 1 << 20

    def __init__(self, runtime: Runtime, config: Config, tuning: dict[str, int] | None = None) -> None:
        super().__init__(runtime, config, tuning)
        self.mask_seconds = 0.0

    def run(self, batch: Prepared, output_cap: int = 8192) -> dict[str, Any]:
        result = super().run(batch, output_cap)
        result['matching_layout'] = 'residue-bitset-batch'
        result['prefilter_build_seconds'] = self.last_stats.get('bounds_ms', 0.0) / 1000
        return result

    def run_lease(self, af: GPUFocus, bf: GPUFocus, first: int, end: int, width: int,
                  output_cap: int = 8192) -> dict[str, Any]:
        """Windows, bounds and the fused kernel for a whole lease in one call; returns the raw
        per-subtile counters, envelope sizes and sorted per-subtile outputs."""
        ng = len(self.filter_groups)
        nt = (end - first + width - 1) // width
        counts = np.zeros(nt * (ng + 3), dtype=np.uint64)
        geometry = np.zeros(2 * nt, dtype=np.uint64)
        n_out = ctypes.c_uint64()
        stats = N.Stats()
        c = self.config
        capacity = min(nt * output_cap, self.lease_output_records)
        for attempt in range(2):
            records = np.zeros(2 * max(1, capacity), dtype=np.uint64)
            self.runtime.check()
            code = self.runtime.lib.pc_run_lease(
                self.runtime.ctx, af.handle, bf.handle, self.filters.handle, ctypes.byref(self.tuning), first,
                end, width, c.lo & MASK, c.lo >> 64, c.hi & MASK, c.hi >> 64, counts, geometry, records,
                capacity, ctypes.byref(n_out), ctypes.byref(stats))
            if code != N.PC_OVERFLOW:
                break
            # counters are complete on overflow: fail like the reference only if a subtile exceeds
            # its cap, otherwise rerun once with room for every record
            if np.any(counts.reshape(nt, ng + 3)[:, ng + 1] > output_cap) or attempt:
                raise OverflowError('lease output overflow; no truncated coverage')
            capacity = int(n_out.value)
        self.runtime.call(code)
        self.runtime.check()
        self.last_stats = stats.as_dict()
        return dict(counts=counts.reshape(nt, ng + 3), geometry=geometry.reshape(nt, 2),
                    per_tile=split_outputs(records[:2 * n_out.value].reshape(-1, 2), nt), stats=self.last_stats)


def compare(reference: dict[str, Any], actual: dict[str, Any]) -> None:
    for key in ('focus_u', 'focus_v', 'cartesian_opportunities', 'valid_focused_candidates', 'genuine_cubes',
                'local_survivors', 'cube_checks', 'filter_groups', 'group_survivors', 'subtile_scopes',
                'cpu_confirmed_hits'):
        if reference[key] != actual[key]:
            raise ArithmeticError('batch/reference mismatch: ' + key)
    if sorted(reference['all_values']) != sorted(actual['all_values']):
        raise ArithmeticError('complete output mismatch')


__all__ = ['Prepared', 'tile_ranges', 'prepare_arrays', 'prepare', 'CachedMatcher', 'FusedMatcher',
           'MaskedMatcher', 'compare', 'launch_plan']
