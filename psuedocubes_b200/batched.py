"""Batched uneven windows: many focus windows with different prime bounds in one launch sequence.

The reference runs one tile (``Matcher.tile``, pseudocube/gpu.py:212-234) or one batch
(``MaskedMatcher.run``, pseudocube/batch_experiment.py:239-248) per call.  Here a whole set of
windows, each ``Window(p, first, end)`` with its own canonical v range and prime bound, is planned
once (``WindowBatch``) and executed by one sequence of launches over the device-resident wheel
tables: the u and v windows of every window are generated together, and stages 2 and 3 treat each
window as a segment with its own interval, subtile width and residual filter family.  The
sequence can be recorded into a CUDA graph and replayed (``run(graph=True)``).

Per window, results carry the keys of the reference's plain tile path (``valid_focused_candidates``,
``group_survivors``, ``all_values``, ``genuine_cubes``, ``cpu_confirmed_hits``, ``subtile_scopes``)
and are identical to the plain per-tile loop over the same v range (``run_production.
compute_batch``), whatever the subtile width: populations are sums over subtiles and outputs are
the complete survivor set.

``Autotuner`` picks the subtile width, the bitset tier (filters and block words), the threads per
CTA and the survivor-buffer size for a workload by timing graph replays, and persists its choice
per device and workload signature.
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os
import random
import time
from concurrent.futures import Future, ThreadPoolExecutor
from dataclasses import dataclass, field
from pathlib import Path
from typing import Any, Iterable, Iterator

import numpy as np

from . import _native as N
from .accounting import EMPTY_DIGEST, digest
from .batch_experiment import verify_values
from .focus import A619, B619, Config
from .gpu import MASK, Filters, GPUFocus, Runtime

#: Prime bounds of the batched workload: the primes in [499, 619] that the reference accepts
#: (``validate_p`` requires p = 1 mod 3).
WORKLOAD_PRIMES = (499, 523, 541, 547, 571, 577, 601, 607, 613, 619)
PRODUCTION_LO, PRODUCTION_HI = 10**27, 3 * 10**27


@dataclass(frozen=True)
class Window:
    """One window: canonical v range [first, end) at prime bound p over (lo, hi], focus (A, B)."""
    p: int
    first: int
    end: int
    lo: int = PRODUCTION_LO
    hi: int = PRODUCTION_HI
    A: int = A619
    B: int = B619

    def config(self) -> Config:
        return Config(self.p, self.lo, self.hi, self.A, self.B)


def seeded_windows(count: int = 512, seed: int = 619003, span_exp: tuple[float, float] = (6.0, 10.0),
                   primes: Iterable[int] = WORKLOAD_PRIMES) -> list[Window]:
    """The batched workload: spans floor(10^U(lo, hi)) v, first uniform in [0, B - span), p uniform
    over ``primes``, production interval and focus."""
    rng = random.Random(seed)
    choices = list(primes)
    out = []
    for _ in range(count):
        span = int(10 ** rng.uniform(*span_exp))
        first = rng.randrange(0, B619 - span)
        out.append(Window(rng.choice(choices), first, first + span))
    return out


class BatchedEngine:
    """Device-resident focus tables and filter families shared by every window batch of a runtime."""

    def __init__(self, runtime: Runtime) -> None:
        self.runtime = runtime
        self._foci: dict[Any, GPUFocus] = {}
        self._families: dict[tuple[int, int, int], Filters] = {}
        self._pairs: dict[tuple[int, int], tuple[GPUFocus, GPUFocus]] = {}
        self._configs: dict[tuple[int, ...], Config] = {}
        self._records = np.empty(0, dtype=np.uint64)

    def record_buffer(self, records: int) -> np.ndarray:
        """A host buffer for ``records`` output records, kept and reused by every batch (results are
        copied out of it), so no step allocates and faults in a fresh output-sized array."""
        if self._records.size < 2 * records:
            self._records = np.empty(2 * records, dtype=np.uint64)
        return self._records

    def focus(self, focus: Any) -> GPUFocus:
        key = (focus.modulus, focus.rings)
        if key not in self._foci:
            self._foci[key] = GPUFocus(self.runtime, focus)
        return self._foci[key]

    def focus_pair(self, config: Config) -> tuple[GPUFocus, GPUFocus]:
        """Device focus tables of (A, B): they depend on A and B only (coefficient-adjusted rings)."""
        key = (config.A, config.B)
        pair = self._pairs.get(key)
        if pair is None:
            af, bf = config.focuses()
            pair = self._pairs[key] = (self.focus(af), self.focus(bf))
        return pair

    def config(self, w: 'Window') -> Config:
        key = (w.p, w.lo, w.hi, w.A, w.B)
        c = self._configs.get(key)
        if c is None:
            if len(self._configs) > 4096:
                self._configs.clear()
            c = self._configs[key] = w.config()
        return c

    def family(self, config: Config) -> Filters:
        key = (config.p, config.A, config.B)
        if key not in self._families:
            self._families[key] = Filters(self.runtime, config)
        return self._families[key]

    def plan(self, windows: list[Window], width: int | None = 100_000_000, tuning: dict[str, int] | None = None,
             output_cap: int = 1 << 16) -> 'WindowBatch':
        """Plan a window batch; width None gives every window a single subtile."""
        return WindowBatch(self, windows, width, tuning, output_cap)

    def stream(self, window_sets: Iterable[list[Window]], width: int | None = 100_000_000,
               tuning: dict[str, int] | None = None, output_cap: int = 1 << 16,
               graph: bool = False) -> Iterator[list[dict[str, Any]]]:
        """The results of consecutive window sets, in order.  One device thread plans, runs and
        copies back set k + 1 while the caller's thread assembles and verifies the results of set
        k, so the host work overlaps the device work; every library call stays on the device
        thread.  A consumer that stops early lets the set in flight finish first."""
        def device(windows: list[Window]) -> tuple['WindowBatch', tuple[np.ndarray, np.ndarray, np.ndarray]]:
            batch = self.plan(windows, width, tuning, output_cap)
            try:
                batch.run(graph=graph)
                return batch, batch.raw()
            finally:
                batch.close()

        pool = ThreadPoolExecutor(1)
        pending: Future | None = None
        try:
            for windows in window_sets:
                upcoming = pool.submit(device, list(windows))
                if pending is not None:
                    batch, raw = pending.result()
                    pending = None
                    yield batch.assemble(*raw)
                pending = upcoming
            if pending is not None:
                batch, raw = pending.result()
                pending = None
                yield batch.assemble(*raw)
        finally:
            pool.shutdown(wait=True)


def _tuning(settings: dict[str, int] | None) -> N.Tuning:
    t = N.Tuning()
    for key, value in (settings or {}).items():
        if key in ('bitset_filters', 'block_words', 'v_chunk', 'threads', 'deep_records'):
            setattr(t, key, int(value))
    return t


class WindowBatch:
    """A planned multi-window launch (pc_multi) with its device buffers."""

    def __init__(self, engine: BatchedEngine, windows: list[Window], width: int | None,
                 tuning: dict[str, int] | None, output_cap: int) -> None:
        if not windows:
            raise ValueError('empty window batch')
        if width is not None and width <= 0:
            raise ValueError('subtile width must be positive')
        rt = engine.runtime
        self.runtime, self.engine, self.windows = rt, engine, list(windows)
        self.widths = [int(width) if width is not None else max(1, w.end - w.first) for w in self.windows]
        self.width = width
        self.output_cap = int(output_cap)
        self.configs = [engine.config(w) for w in self.windows]
        foci: list[GPUFocus] = []
        families: list[Filters] = []
        index_f: dict[int, int] = {}
        index_m: dict[int, int] = {}
        self._family_of = []
        spec = (N.Window * len(self.windows))()
        for i, (w, c) in enumerate(zip(self.windows, self.configs)):
            if not 0 <= w.first < w.end <= c.B:
                raise ValueError('window outside the canonical domain')
            ids = []
            for g in engine.focus_pair(c):
                k = index_f.get(id(g))
                if k is None:
                    k = index_f[id(g)] = len(foci)
                    foci.append(g)
                ids.append(k)
            fam = engine.family(c)
            m = index_m.get(id(fam))
            if m is None:
                m = index_m[id(fam)] = len(families)
                families.append(fam)
            self._family_of.append(m)
            s = spec[i]
            s.first, s.end, s.width = w.first, w.end, self.widths[i]
            s.lo0, s.lo1, s.hi0, s.hi1 = c.lo & MASK, c.lo >> 64, c.hi & MASK, c.hi >> 64
            s.focus_a, s.focus_b, s.family = ids[0], ids[1], m
        self.foci, self.families = foci, families
        focus_ptrs = (ctypes.c_void_p * len(foci))(*[g.handle.value for g in foci])
        family_ptrs = (ctypes.c_void_p * len(families))(*[f.handle.value for f in families])
        self.tuning = _tuning(tuning)
        handle = ctypes.c_void_p()
        rt.check()
        rt.call(rt.lib.pc_multi_create(rt.ctx, focus_ptrs, len(foci), family_ptrs, len(families), spec,
                                       len(self.windows), ctypes.byref(self.tuning), self.output_cap,
                                       ctypes.byref(handle)))
        self.handle = handle
        n = len(self.windows)
        self.tile_base = np.zeros(n + 1, dtype=np.uint32)
        self.sizes = np.zeros(2 * n, dtype=np.uint64)
        info = np.zeros(8, dtype=np.uint64)
        rt.lib.pc_multi_layout(handle, self.tile_base, self.sizes, info)
        self.ntiles, self.stride = int(info[0]), int(info[1])
        self.layout = dict(subtiles=self.ntiles, stride=self.stride, u_entries=int(info[2]), v_entries=int(info[3]),
                           deep_records=int(info[4]), bitset_filters=int(info[5]), block_words=int(info[6]),
                           threads=int(info[7]))
        self.last_stats: dict[str, Any] = {}

    def run(self, graph: bool = False) -> dict[str, Any]:
        """Execute every window on the device (eager, or replay of the recorded graph) and return the
        raw counters; ``results()`` turns them into per-window result dicts."""
        rt = self.runtime
        stats = N.Stats()
        rt.check()
        rt.call(rt.lib.pc_multi_run(rt.ctx, self.handle, N.PC_RUN_GRAPH if graph else 0, ctypes.byref(stats)))
        self.last_stats = stats.as_dict()
        return self.last_stats

    def raw(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        rt = self.runtime
        counts = np.empty(max(1, self.ntiles * self.stride), dtype=np.uint64)     # every entry is written
        geometry = np.empty(max(2, 2 * self.ntiles), dtype=np.uint64)
        records = self.engine.record_buffer(max(1, self.output_cap))
        n_out = ctypes.c_uint64()
        rt.call(rt.lib.pc_multi_results(rt.ctx, self.handle, counts, geometry, records, self.output_cap,
                                        ctypes.byref(n_out)))
        return (counts[:self.ntiles * self.stride].reshape(self.ntiles, self.stride),
                geometry[:2 * self.ntiles].reshape(self.ntiles, 2), records[:2 * n_out.value].reshape(-1, 2).copy())

    def positions(self) -> int:
        """Focused candidate positions of the last run (all windows)."""
        counts, _, _ = self.raw()
        return int(counts[:, 0].sum())

    def results(self) -> list[dict[str, Any]]:
        """Per-window results of the last run, host-verified like the reference's tile results
        (the fields of batch_experiment.batch_result)."""
        return self.assemble(*self.raw())

    def assemble(self, counts: np.ndarray, geometry: np.ndarray, records: np.ndarray) -> list[dict[str, Any]]:
        """Per-window results from the raw counters, envelope sizes and output records of a run
        (host work only).  The subtile fields of all windows are formed in a few array passes and
        one pass over the subtiles; only subtiles that emitted values are visited one by one."""
        n, nt = len(self.windows), self.ntiles
        tb = self.tile_base.astype(np.int64)
        per = np.diff(tb)
        ngs = [self.families[self._family_of[i]].ng for i in range(n)]
        tile_ng = np.repeat(np.array(ngs, dtype=np.int64), per)
        at = np.arange(nt)
        emitted = counts[at, tile_ng + 1]
        if np.any(counts[at, tile_ng + 2]):
            raise ArithmeticError('unsigned underflow')
        tile = (records[:, 1] >> np.uint64(32)).astype(np.int64)
        if len(tile) and (tile.min() < 0 or tile.max() >= nt):
            raise ArithmeticError('output record outside the launch')
        if not np.array_equal(np.bincount(tile, minlength=nt), emitted.astype(np.int64)):
            raise ArithmeticError('device output count disagrees with its records')
        order = np.argsort(tile, kind='stable')
        tile_sorted = tile[order]
        lo_limb, hi_limb = records[order, 0], records[order, 1] & np.uint64(0xFFFFFFFF)
        cuts = np.searchsorted(tile_sorted, np.arange(nt + 1)).tolist()
        # subtile bounds: window first + k * width, the last one ending at the window's end
        owner = np.repeat(np.arange(n), per)
        firsts = [w.first for w in self.windows]
        ends = [w.end for w in self.windows]
        if max(ends, default=0) + max(self.widths, default=0) < 2**63:
            f64, w64 = np.array(firsts, dtype=np.int64)[owner], np.array(self.widths, dtype=np.int64)[owner]
            sub_first = f64 + (at - tb[owner]) * w64
            sub_end = np.minimum(sub_first + w64, np.array(ends, dtype=np.int64)[owner])
            first_l, end_l = sub_first.tolist(), sub_end.tolist()
        else:                                             # bounds beyond 64 bits: plain integers
            first_l, end_l = [], []
            for w, wd in zip(self.windows, self.widths):
                for a in range(w.first, w.end, wd):
                    first_l.append(a)
                    end_l.append(min(a + wd, w.end))
        starts, stops = list(map(str, first_l)), list(map(str, end_l))
        valid = counts[:, 0].tolist()
        emitted_list = emitted.tolist()
        sums = np.add.reduceat(counts, tb[:-1], axis=0).tolist() if nt else [[0] * self.stride] * n
        gu, gv = geometry[:, 0].tolist(), geometry[:, 1].tolist()
        cart = [a * b for a, b in zip(gu, gv)]
        # group populations per subtile, one conversion per family over the family's subtiles
        groups: list = [None] * nt
        fam_of_tile = np.repeat(np.array(self._family_of, dtype=np.int64), per)
        for f in sorted(set(self._family_of)):
            idx = np.nonzero(fam_of_tile == f)[0]
            for t, row in zip(idx.tolist(), counts[idx, 1:self.families[f].ng + 1].tolist()):
                groups[t] = row
        # emitted values: sorted per subtile, checked against the subtile, digested
        digests = [EMPTY_DIGEST] * nt
        values_of: dict[int, list[int]] = {}
        for t in np.nonzero(emitted)[0].tolist():
            k0, k1 = cuts[t], cuts[t + 1]
            tile_values = sorted(int(a) | int(b) << 64 for a, b in zip(lo_limb[k0:k1].tolist(), hi_limb[k0:k1].tolist()))
            i = int(owner[t])
            c, first, end = self.configs[i], first_l[t], end_l[t]
            if any(not first <= c.canonical(x)[1] < end for x in tile_values):
                raise ArithmeticError('output assigned to wrong subtile')
            digests[t] = digest([str(x) for x in tile_values])
            values_of.setdefault(i, []).extend(tile_values)
        scopes = [{'first': a, 'end': b, 'valid_focused_candidates': v, 'group_survivors': g, 'local_survivors': e,
                   'output_sha256': d}
                  for a, b, v, g, e, d in zip(starts, stops, valid, groups, emitted_list, digests)]
        tbl, sizes = tb.tolist(), self.sizes.tolist()
        out = []
        for i, (w, c) in enumerate(zip(self.windows, self.configs)):
            t0, t1, ng = tbl[i], tbl[i + 1], ngs[i]
            values = values_of.get(i, [])
            hits = verify_values(c, values) if values else []
            row = dict(status='PASS', host_verified=True, focus_u=int(sizes[2 * i]),
                       focus_v=int(sizes[2 * i + 1]), cartesian_opportunities=sum(cart[t0:t1]),
                       valid_focused_candidates=sum(valid[t0:t1]), genuine_cubes=len(values) - len(hits),
                       local_survivors=len(values), cube_checks=len(values), subtile_scopes=scopes[t0:t1],
                       filter_groups=self.families[self._family_of[i]].filter_groups,
                       group_survivors=sums[i][1:ng + 1] if t1 > t0 else [0] * ng,
                       all_values=[str(x) for x in values], cpu_confirmed_hits=hits, overflow_splits=[],
                       p=w.p, first=str(w.first), end=str(w.end))
            out.append(row)
        return out

    def close(self) -> None:
        if getattr(self, 'handle', None) and self.runtime.ctx:
            self.runtime.lib.pc_multi_free(self.runtime.ctx, self.handle)
            self.handle = None

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------------------------------
# autotuner

#: the autotuner's choice for the 512 seeded uneven windows (p in [499, 619]) on a B200; a batch
#: whose deep survivors outgrow deep_records per CTA is rerun larger when it runs eagerly
DEFAULT_SETTINGS: dict[str, int] = dict(width=1 << 27, bitset_filters=7, block_words=32, threads=896, deep_records=8192)
SEARCH_SPACE: dict[str, tuple[int, ...]] = dict(
    width=(1 << 20, 1 << 22, 1 << 24, 1 << 26, 1 << 27),
    bitset_filters=(5, 6, 7, 8),
    block_words=(16, 32, 64),
    threads=(512, 768, 896, 1024),
)


def workload_signature(windows: list[Window]) -> str:
    """Coarse description of a workload, stable across seeds of the same distribution."""
    spans = sorted(w.end - w.first for w in windows)
    total = sum(spans)
    ps = sorted({w.p for w in windows})
    return f'n{len(windows)}-span{len(str(total))}-median{len(str(spans[len(spans) // 2]))}-p{ps[0]}-{ps[-1]}'


def tuning_path() -> Path:
    env = os.environ.get('PSUEDOCUBES_TUNING')
    if env:
        return Path(env)
    return Path.home() / '.cache' / 'psuedocubes_b200' / 'tuning.json'


@dataclass
class TuneResult:
    settings: dict[str, int]
    ms: float
    trials: list[dict[str, Any]] = field(default_factory=list)


class Autotuner:
    """Coordinate search over subtile width, bitset filters, block words and threads, timed by
    graph replays; the survivor buffer is then sized from the measured deep-survivor peak."""

    def __init__(self, engine: BatchedEngine, path: Path | None = None, replays: int = 3) -> None:
        self.engine, self.path, self.replays = engine, path or tuning_path(), replays

    def key(self, windows: list[Window]) -> str:
        return f'{self.engine.runtime.device_name}|{workload_signature(windows)}'

    def load(self, windows: list[Window]) -> dict[str, int] | None:
        try:
            return json.loads(self.path.read_text()).get(self.key(windows))
        except (OSError, ValueError):
            return None

    def save(self, windows: list[Window], settings: dict[str, int]) -> None:
        try:
            table = json.loads(self.path.read_text())
        except (OSError, ValueError):
            table = {}
        table[self.key(windows)] = settings
        self.path.parent.mkdir(parents=True, exist_ok=True)
        self.path.write_text(json.dumps(table, indent=1, sort_keys=True))

    def measure(self, windows: list[Window], settings: dict[str, int], output_cap: int) -> tuple[float, int]:
        tuning = {k: v for k, v in settings.items() if k != 'width'}
        batch = self.engine.plan(windows, settings['width'], tuning, output_cap)
        try:
            batch.run(graph=True)                         # eager run, capture, first replay
            best = min(batch.run(graph=True)['kernel_ms'] for _ in range(self.replays))
            return best, int(batch.last_stats.get('deep_survivors', 0))
        finally:
            batch.close()

    def tune(self, windows: list[Window], output_cap: int = 1 << 16, reuse: bool = True) -> TuneResult:
        if reuse:
            known = self.load(windows)
            if known:
                return TuneResult(dict(known), float('nan'))
        best = dict(DEFAULT_SETTINGS)
        best_ms, deep = self.measure(windows, best, output_cap)
        trials = [dict(best, ms=best_ms)]
        for knob, values in SEARCH_SPACE.items():
            for value in values:
                if value == best[knob]:
                    continue
                trial = dict(best, **{knob: value})
                try:
                    ms, d = self.measure(windows, trial, output_cap)
                except (ValueError, MemoryError) as exc:
                    trials.append(dict(trial, error=str(exc)))
                    continue
                trials.append(dict(trial, ms=ms))
                if ms < best_ms:
                    best, best_ms, deep = trial, ms, d
        # survivor buffer: the measured per-CTA peak with headroom, as a power of two
        best['deep_records'] = max(1024, 1 << int(max(deep, 1) * 2 - 1).bit_length())
        self.save(windows, best)
        return TuneResult(best, best_ms, trials)


def workload_digest(windows: list[Window]) -> str:
    h = hashlib.sha256()
    for w in windows:
        h.update(f'{w.p},{w.first},{w.end},{w.lo},{w.hi},{w.A},{w.B};'.encode())
    return h.hexdigest()


__all__ = ['Window', 'WORKLOAD_PRIMES', 'seeded_windows', 'BatchedEngine', 'WindowBatch', 'Autotuner',
           'DEFAULT_SETTINGS', 'SEARCH_SPACE', 'workload_signature', 'workload_digest', 'tuning_path']
