"""Lease execution and compact, reproducible lease receipts.

Mirrors pseudocube/optimized.py:15-90 (PROFILE, BATCH_WIDTH, LEASE_WIDTH, Accumulator,
compute_lease).  ``compute_lease`` runs a whole lease through one device call when the matcher
offers it (windows of both focuses generated once for the lease from the resident wheels, then the
fused kernel over all 16,384 subtiles), and folds the per-batch results into the Accumulator in
batch order, so the transcript is byte-identical to a batch-by-batch run.
"""
from __future__ import annotations

import ctypes
import hashlib
import time
from collections import deque
from concurrent.futures import Future, ThreadPoolExecutor
from typing import Any, Callable, Iterable, Iterator

import numpy as np

from .accounting import EMPTY_DIGEST, digest, encoded_scopes
from . import _native as N
from .batch_experiment import MaskedMatcher, batch_result, prepare, split_outputs, verify_values
from .focus import Tile
from .gpu import MASK, GPUFocus
from .multi import validate_result

PROFILE: dict[str, Any] = dict(engine='residue-bitset-batch-v1', tile_width=100_000_000,
                               tiles_per_compute_batch=64, compute_batches_per_lease=256,
                               receipt_storage='sqlite-gzip', receipt_format='compact-batch-v1',
                               authorization='Deploy to production')
BATCH_WIDTH = PROFILE['tile_width'] * PROFILE['tiles_per_compute_batch']
LEASE_WIDTH = BATCH_WIDTH * PROFILE['compute_batches_per_lease']
COUNTS = ('focus_u', 'focus_v', 'cartesian_opportunities', 'valid_focused_candidates',
          'genuine_cubes', 'local_survivors', 'cube_checks')
TIMINGS = ('kernel_seconds', 'focus_enumeration_seconds', 'transfer_seconds',
           'verification_seconds', 'prefilter_build_seconds')


class Accumulator:
    """Contiguous batches of one lease folded into a compact receipt."""

    def __init__(self, first: int, end: int) -> None:
        if not 0 <= first < end or end - first > LEASE_WIDTH:
            raise ValueError('invalid optimized lease')
        self.first, self.end, self.cursor = first, end, first
        self.counts = dict.fromkeys(COUNTS, 0)
        self.timings = dict.fromkeys(TIMINGS, 0.0)
        self.values: list[str] = []
        self.hits: list[dict[str, Any]] = []
        self.groups: list[int] = []
        self.filters: list[list[int]] | None = None
        self.transcript = hashlib.sha256()
        self.batches = self.subtiles = 0

    def add(self, first: int, end: int, row: dict[str, Any]) -> None:
        if first != self.cursor or end != min(first + BATCH_WIDTH, self.end):
            raise ValueError('gap, overlap or changed compute batch geometry')
        validate_result(first, end, row)
        width = PROFILE['tile_width']
        expected = [(v, min(v + width, end)) for v in range(first, end, width)]
        actual = [(int(s['first']), int(s['end'])) for s in row['subtile_scopes']]
        if actual != expected:
            raise ValueError('changed arithmetic subtile geometry')
        if self.filters is None:
            self.filters = [list(group) for group in row['filter_groups']]
            self.groups = [0] * len(self.filters)
        if row['filter_groups'] != self.filters or len(row['group_survivors']) != len(self.groups):
            raise ValueError('residue filters changed during execution')
        for key in COUNTS:
            self.counts[key] += int(row[key])
        for key in TIMINGS:
            self.timings[key] += float(row.get(key, 0.0))
        for i, count in enumerate(row['group_survivors']):
            self.groups[i] += int(count)
        self.values.extend(row['all_values'])
        self.hits.extend(row['cpu_confirmed_hits'])
        self.transcript.update(encoded_scopes(row['subtile_scopes']))
        self.batches += 1
        self.subtiles += len(actual)
        self.cursor = end

    def finish(self, seconds: float) -> dict[str, Any]:
        if self.cursor != self.end:
            raise ValueError('unfinished lease cannot become coverage')
        row = dict(status='PASS', host_verified=True, receipt_format=PROFILE['receipt_format'],
                   tile_width=PROFILE['tile_width'], compute_batch_width=BATCH_WIDTH,
                   compute_batches=self.batches, subtiles_executed=self.subtiles,
                   subtile_scopes=[dict(first=str(self.first), end=str(self.end),
                                        transcript_sha256=self.transcript.hexdigest(),
                                        output_sha256=digest(self.values))],
                   **self.counts, **self.timings, group_survivors=self.groups, filter_groups=self.filters,
                   all_values=self.values, cpu_confirmed_hits=self.hits, overflow_splits=[],
                   elapsed_seconds=seconds,
                   claim='Executed primary coverage; independent arithmetic replay required before any minimum claim.')
        validate_result(self.first, self.end, row)
        return row


def lease_batches(matcher: MaskedMatcher, af: GPUFocus, bf: GPUFocus, first: int, end: int) -> list[tuple[int, int, dict[str, Any]]]:
    """Every batch result of [first, end) from one fused lease call, in batch order."""
    width = PROFILE['tile_width']
    Tile(first, end).validate(matcher.config)
    raw = matcher.run_lease(af, bf, first, end, width)
    stats = raw['stats']
    nbatches = (end - first + BATCH_WIDTH - 1) // BATCH_WIDTH
    out = []
    for k in range(nbatches):
        start = first + k * BATCH_WIDTH
        stop = min(start + BATCH_WIDTH, end)
        # subtile bounds only: batch_result reads (first, end) and the lease call already checked
        # the geometry on the device
        ranges = [(v, min(v + width, stop), 0, 0) for v in range(start, stop, width)]
        t0 = k * PROFILE['tiles_per_compute_batch']
        rows = slice(t0, t0 + len(ranges))
        geometry = [(int(a), int(b)) for a, b in raw['geometry'][rows]]
        verification_started = time.perf_counter()
        row = batch_result(matcher.config, ranges, raw['counts'][rows], raw['per_tile'][rows], geometry,
                           matcher.filter_groups, 8192)
        row.update(kernel_seconds=stats['kernel_ms'] / 1000 / nbatches,
                   focus_enumeration_seconds=stats['window_ms'] / 1000 / nbatches,
                   prefilter_build_seconds=stats['bounds_ms'] / 1000 / nbatches, transfer_seconds=0.0,
                   verification_seconds=time.perf_counter() - verification_started,
                   matching_layout='residue-bitset-lease')
        out.append((start, stop, row))
    return out


def lease_receipt(matcher: MaskedMatcher, raw: dict[str, Any], first: int, end: int, started: float) -> dict[str, Any]:
    """The compact receipt of a whole-lease device call, built from its counter arrays: the same
    fields, sums and transcript bytes as folding every batch result into an Accumulator, with the
    canonical JSON of the 16,384 subtile scopes written by the library (pc_scopes_json) instead of
    through 16,384 dicts.  Every emitted value is re-verified on the host as in batch_result."""
    config, width = matcher.config, PROFILE['tile_width']
    if not 0 <= first < end or end - first > LEASE_WIDTH:
        raise ValueError('invalid optimized lease')
    counts, geometry, per_tile, stats = raw['counts'], raw['geometry'], raw['per_tile'], raw['stats']
    nt, ng = counts.shape[0], len(matcher.filter_groups)
    if nt != (end - first + width - 1) // width:
        raise ValueError('changed arithmetic subtile geometry')
    if np.any(counts[:, ng + 2]):
        raise ArithmeticError('unsigned underflow')
    if np.any(counts[:, ng + 1] > 8192):
        raise OverflowError('fused tile output overflow; no truncated coverage')
    verification_started = time.perf_counter()
    digests = [EMPTY_DIGEST] * nt
    values: list[int] = []
    emitted = counts[:, ng + 1].tolist()
    for t in np.nonzero(counts[:, ng + 1])[0].tolist():
        tile_values = per_tile[t]
        lo = first + t * width
        if len(tile_values) != emitted[t]:
            raise ArithmeticError('device output count disagrees with its records')
        if any(not lo <= config.canonical(n)[1] < min(lo + width, end) for n in tile_values):
            raise ArithmeticError('output assigned to wrong subtile')
        digests[t] = digest([str(n) for n in tile_values])
        values.extend(tile_values)
    if sum(emitted) != len(values):
        raise ArithmeticError('device output count disagrees with its records')
    hits = verify_values(config, values)
    lib = matcher.runtime.lib
    text = ''.join(digests).encode()
    cap = nt * (260 + 21 * ng) + 64
    buf = np.empty(cap, dtype=np.uint8)                  # written by the library, not zeroed first
    size = ctypes.c_uint64()
    code = lib.pc_scopes_json(np.ascontiguousarray(counts, dtype=np.uint64).reshape(-1), counts.shape[1], ng, nt, first,
                              end, width, PROFILE['tiles_per_compute_batch'], text, buf.ctypes.data, cap,
                              ctypes.byref(size))
    if code:
        raise RuntimeError(f'scope encoding failed ({code})')
    transcript = hashlib.sha256(memoryview(buf)[:size.value]).hexdigest()
    verification_seconds = time.perf_counter() - verification_started
    gu, gv = geometry[:, 0], geometry[:, 1]
    if nt and int(gu.max()) * int(gv.max()) * nt < 1 << 64:      # the uint64 sum is exact
        cartesian = int((gu * gv).sum())
    else:
        cartesian = int(sum(gu.astype(object) * gv.astype(object)))
    strs = [str(n) for n in values]
    nbatches = (end - first + BATCH_WIDTH - 1) // BATCH_WIDTH
    row = dict(status='PASS', host_verified=True, receipt_format=PROFILE['receipt_format'],
               tile_width=width, compute_batch_width=BATCH_WIDTH, compute_batches=nbatches, subtiles_executed=nt,
               subtile_scopes=[dict(first=str(first), end=str(end), transcript_sha256=transcript,
                                    output_sha256=digest(strs))],
               focus_u=int(geometry[:, 0].sum()), focus_v=int(geometry[:, 1].sum()),
               cartesian_opportunities=cartesian, valid_focused_candidates=int(counts[:, 0].sum()),
               genuine_cubes=len(values) - len(hits), local_survivors=len(values), cube_checks=len(values),
               kernel_seconds=stats['kernel_ms'] / 1000, focus_enumeration_seconds=stats['window_ms'] / 1000,
               transfer_seconds=0.0, verification_seconds=verification_seconds,
               prefilter_build_seconds=stats['bounds_ms'] / 1000,
               group_survivors=[int(n) for n in counts[:, 1:ng + 1].sum(axis=0)],
               filter_groups=[list(g) for g in matcher.filter_groups], all_values=strs, cpu_confirmed_hits=hits,
               overflow_splits=[], elapsed_seconds=time.monotonic() - started,
               claim='Executed primary coverage; independent arithmetic replay required before any minimum claim.')
    validate_result(first, end, row)
    return row


def compute_lease(matcher: MaskedMatcher, af: GPUFocus, bf: GPUFocus, first: int, end: int,
                  heartbeat: Callable[[], None] = lambda: None) -> dict[str, Any]:
    started = time.monotonic()
    acc = Accumulator(first, end)
    if hasattr(matcher, 'run_lease'):
        Tile(first, end).validate(matcher.config)
        raw = matcher.run_lease(af, bf, first, end, PROFILE['tile_width'])
        heartbeat()
        return lease_receipt(matcher, raw, first, end, started)
    else:
        for start in range(first, end, BATCH_WIDTH):
            stop = min(start + BATCH_WIDTH, end)
            batch = prepare(matcher.runtime, matcher.config, af, bf, start, stop, PROFILE['tile_width'])
            acc.add(start, stop, matcher.run(batch))
            heartbeat()
    return acc.finish(time.monotonic() - started)


class _LeaseChunk:
    """Host buffers for up to ``size`` leases of one ``pc_run_leases`` call, reused chunk after
    chunk (the receipts copy everything they keep out of them)."""

    def __init__(self, matcher: MaskedMatcher, size: int, width: int, output_records: int) -> None:
        self.matcher, self.size, self.width, self.records = matcher, size, width, output_records
        self.stride = len(matcher.filter_groups) + 3
        ntmax = (LEASE_WIDTH + width - 1) // width
        # page-locked: the library's device-to-host copies at the end of each lease run at full speed
        self.counts = [N.pinned(ntmax * self.stride) for _ in range(size)]
        self.geometry = [N.pinned(2 * ntmax) for _ in range(size)]
        self.out = [np.zeros(2 * output_records, dtype=np.uint64) for _ in range(size)]
        self.n_out = np.zeros(size, dtype=np.uint64)
        self.stats = (N.Stats * size)()
        self.status = np.zeros(size, dtype=np.int32)
        self.leases: list[tuple[int, int, float]] = []
        self.future: Future | None = None

    def submit(self, pool: ThreadPoolExecutor, af: GPUFocus, bf: GPUFocus, leases: list[tuple[int, int]]) -> None:
        m, c = self.matcher, self.matcher.config
        self.leases = [(first, end, time.monotonic()) for first, end in leases]
        self.status[:] = 0
        self.n_out[:] = 0
        n = len(leases)
        firsts = np.array([f for f, _ in leases], dtype=np.uint64)
        ends = np.array([e for _, e in leases], dtype=np.uint64)
        ptrs = lambda arrays: (ctypes.c_void_p * n)(*[x.ctypes.data for x in arrays[:n]])
        args = (m.runtime.ctx, af.handle, bf.handle, m.filters.handle, ctypes.byref(m.tuning), n, firsts, ends,
                self.width, c.lo & MASK, c.lo >> 64, c.hi & MASK, c.hi >> 64, ptrs(self.counts), ptrs(self.geometry),
                ptrs(self.out), self.records, self.n_out, self.stats, self.status)

        def run() -> int:
            m.runtime.check()
            return m.runtime.lib.pc_run_leases(*args)

        self.future = pool.submit(run)

    def wait(self, i: int) -> int:
        """The return code of lease i, once its results are on the host."""
        while self.status[i] == 0 and not self.future.done():
            time.sleep(0.0002)
        if self.status[i] == 0:                       # the call ended before lease i: its own failure
            code = self.future.result()
            self.matcher.runtime.call(code, 'lease list')
            raise RuntimeError(f'lease list stopped before lease {i}')
        return int(self.status[i]) - 1

    def raw(self, i: int) -> dict[str, Any]:
        first, end, _ = self.leases[i]
        nt = (end - first + self.width - 1) // self.width
        n = int(self.n_out[i])
        m = self.matcher
        m.last_stats = self.stats[i].as_dict()
        return dict(counts=self.counts[i][:nt * self.stride].reshape(nt, self.stride),
                    geometry=self.geometry[i][:2 * nt].reshape(nt, 2),
                    per_tile=split_outputs(self.out[i][:2 * n].reshape(-1, 2), nt), stats=m.last_stats)

    def finish(self) -> None:
        self.future.result()


class _LeaseCalls:
    """The same protocol for a matcher with only ``run_lease``: one helper-thread call per lease."""

    def __init__(self, matcher: Any, width: int) -> None:
        self.matcher, self.width = matcher, width
        self.leases: list[tuple[int, int, float]] = []
        self.futures: list[Future] = []

    def submit(self, pool: ThreadPoolExecutor, af: GPUFocus, bf: GPUFocus, leases: list[tuple[int, int]]) -> None:
        self.leases = [(first, end, time.monotonic()) for first, end in leases]
        self.futures = [pool.submit(self.matcher.run_lease, af, bf, first, end, self.width) for first, end in leases]

    def wait(self, i: int) -> int:
        self.futures[i].result()
        return N.PC_OK

    def raw(self, i: int) -> dict[str, Any]:
        return self.futures[i].result()

    def finish(self) -> None:
        for future in self.futures:
            future.result()


def compute_leases(matcher: MaskedMatcher, af: GPUFocus, bf: GPUFocus, leases: Iterable[tuple[int, int]],
                   heartbeat: Callable[[], None] = lambda: None, chunk: int = 4) -> Iterator[dict[str, Any]]:
    """Receipts of a sequence of leases, in order, each identical to ``compute_lease`` of it.

    A worker that runs leases back to back overlaps them.  One helper thread runs the device work:
    ``pc_run_leases`` over ``chunk`` leases at a time, with the next chunk queued behind it, so
    consecutive leases follow each other on the device with no interpreter step between them.
    This thread builds and re-verifies the receipt of each lease as soon as the library marks it
    done.  Every device call goes through the one helper thread, so the library context is never
    used by two threads at once.  A lease that fails in the list (an output buffer too small, say)
    is rerun alone through ``MaskedMatcher.run_lease``, which applies the reference's overflow rule.
    Bounds are validated before a lease is issued."""
    if not hasattr(matcher, 'run_lease'):
        for first, end in leases:
            yield compute_lease(matcher, af, bf, first, end, heartbeat)
        return
    width = PROFILE['tile_width']
    pending = iter(leases)

    def take() -> list[tuple[int, int]]:
        out = []
        for first, end in pending:
            if not 0 <= first < end or end - first > LEASE_WIDTH:
                raise ValueError('invalid optimized lease')
            Tile(first, end).validate(matcher.config)
            out.append((first, end))
            if len(out) == chunk:
                break
        return out

    with ThreadPoolExecutor(max_workers=1) as pool:
        if isinstance(matcher, MaskedMatcher):
            # page-locked buffers are slow to allocate: the matcher keeps its two chunks for later calls
            key = (chunk, width, matcher.lease_output_records)
            kept = getattr(matcher, '_lease_chunks', None)
            if kept is None or kept[0] != key:
                kept = (key, [_LeaseChunk(matcher, chunk, width, matcher.lease_output_records) for _ in range(2)])
                matcher._lease_chunks = kept
            slots = kept[1]
        else:
            slots = [_LeaseCalls(matcher, width) for _ in range(2)]
        running: deque = deque()
        for slot in slots:
            batch = take()
            if batch:
                slot.submit(pool, af, bf, batch)
                running.append(slot)
        while running:
            slot = running[0]
            for i, (first, end, started) in enumerate(slot.leases):
                code = slot.wait(i)
                if code == N.PC_OK:
                    raw = slot.raw(i)
                else:
                    if code != N.PC_OVERFLOW:
                        matcher.runtime.call(code, 'lease')
                    rest = slot.leases[i:]
                    slot.finish()
                    raws = [pool.submit(matcher.run_lease, af, bf, f, e, width) for f, e, _ in rest]
                    for (f, e, t0), fut in zip(rest, raws):
                        result = fut.result()
                        heartbeat()
                        yield lease_receipt(matcher, result, f, e, t0)
                    break
                heartbeat()
                yield lease_receipt(matcher, raw, first, end, started)
            slot.finish()
            running.popleft()
            batch = take()
            if batch:                                 # reuses the buffers of the chunk just consumed
                slot.submit(pool, af, bf, batch)
                running.append(slot)
