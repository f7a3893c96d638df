"""Served range certification: requests (p, x_lo, x_hi) answered by continuous batching.

The reference certifies one fixed geometry, Config(p, lo, hi, A619, B619), batch by batch.  A
request here is an arbitrary interval (x_lo, x_hi] at prime bound p.  With the A619/B619 focus
every request would have to visit all of v in [0, B619) (6.7e12 focus values) however narrow it
is, so each request gets its own focus split (A', B') from ``plan_request``: A' and B' are
products of prefixes of the ring lists of A619 and B619 (9, 2 and primes q = 1 mod 3 only; a ring
q = 2 mod 3 would multiply the focus count by q - 1 for a density gain of (q - 1)/q), chosen by a
device cost model of u entries, v entries and focused positions, under the reference's bound
checks (Config: A', B' < 2^63, u < 2^64, u B' < 2^128).  The output set of a request does not
depend on the split; its populations are those of its own Config.

``ServedLoop`` runs requests as they arrive.  A request is cut into windows (v ranges, and x
sub-ranges when one v row alone would exceed a window's u budget); every GPU step packs windows of
all admitted requests, smallest remaining work first, into one multi-window launch
(``BatchedEngine``), so requests that arrive while others run join the next step and their work
shares the device.  Requests are admitted in arrival order while the device memory they reserve
(their focus tables and output buffers) fits the cap; focus tables and filter families stay
resident across requests.  The host verifies one step's outputs while the device runs the next.
Every finished request is checked against the device genuine-cube control (``cubes``): the cubes
it emitted must be exactly the cubes a^3 in (x_lo, x_hi] with a coprime to every prime <= p.
``plain_loop`` is the sequential plain per-request loop of the same build (the reference's plain
tile matcher, one request after another) used as the baseline.
"""
from __future__ import annotations

import math
import random
import time
from collections import deque
from concurrent.futures import Future, ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import Any

import numpy as np

from .batched import BatchedEngine, Window
from .cubes import genuine_cube_count
from .focus import Config, Tile
from .gpu import Matcher, Runtime
from .tables import allowed
from .verify import MATERIALISE_MAX, VECTOR_MIN, cube_limbs, icbrt_many, verify, verify_many

A_RINGS = (2, 7, 13, 31, 43, 73, 79, 127, 139, 157, 181)   # the rings of A619, ascending
B_RINGS = (9, 19, 37, 61, 67, 97, 103, 109, 151, 163)      # the rings of B619, ascending
SERVED_PRIMES = (499, 523, 541, 547, 571, 577, 601, 607, 613, 619)
X_MAX = 3 * 10**27
#: device seconds per u entry, per v entry and per focused position.  A u entry costs its window
#: generation plus its share of the matcher's fixed per-block work (pattern load, residue rows,
#: barriers: about 30 us of one CTA per 1024-entry block, measured on served steps whose blocks
#: met ~200 v rows each); a v entry its bounds and pieces; a position its share of the bitset tier.
COST_U, COST_V, COST_POSITION = 200e-12, 100e-12, 0.08e-12
U_WINDOW, V_WINDOW, P_WINDOW = 1 << 24, 1 << 22, 2 * 10**10
STEP_U, STEP_V, STEP_P, STEP_WINDOWS = 1 << 27, 1 << 24, 2 * 10**11, 512


@dataclass(frozen=True)
class Request:
    id: int
    p: int
    lo: int          # exclusive
    hi: int          # inclusive
    arrival: float = 0.0


@dataclass(frozen=True)
class Plan:
    a: int
    b: int
    A: int
    B: int
    count_a: int
    count_b: int
    seconds: float    # modelled device time

    @property
    def density_a(self) -> float:
        return self.count_a / self.A

    @property
    def density_b(self) -> float:
        return self.count_b / self.B


def _count(q: int) -> int:
    return len(allowed(q))


def plan_request(p: int, lo: int, hi: int) -> Plan:
    """The focus split of least modelled device time for (lo, hi] (deterministic)."""
    if not 0 <= lo < hi <= X_MAX:
        raise ValueError('invalid interval')
    span = hi - lo
    best: Plan | None = None
    for a in range(1, len(A_RINGS) + 1):
        A = math.prod(A_RINGS[:a])
        ca = math.prod(_count(q) for q in A_RINGS[:a])
        for b in range(1, len(B_RINGS) + 1):
            B = math.prod(B_RINGS[:b])
            if A >= 1 << 63 or B >= 1 << 63 or max(A_RINGS[:a] + B_RINGS[:b]) > p:
                continue
            max_u = (hi + (B - 1) * A) // B
            if max_u >= 1 << 64 or max_u * B >= 1 << 128:
                continue
            cb = math.prod(_count(q) for q in B_RINGS[:b])
            positions = span * (ca / A) * (cb / B)
            sweeps = max(1, math.ceil(span * ca / A / B / (U_WINDOW / 2)))   # x sub-ranges (request_windows)
            u_entries = sweeps * ca + ca * span / (A * B)
            seconds = COST_U * u_entries + COST_V * sweeps * cb + COST_POSITION * positions
            if best is None or seconds < best.seconds:
                best = Plan(a, b, A, B, ca, cb, seconds)
    if best is None:
        raise ValueError('no focus split satisfies the arithmetic bounds')
    return best


def split_plan(p: int, lo: int, hi: int, a: int, b: int) -> Plan:
    """The plan of a given focus split (prefix lengths a of A's rings and b of B's rings)."""
    A, B = math.prod(A_RINGS[:a]), math.prod(B_RINGS[:b])
    Config(p, lo, hi, A, B)                                   # the reference's bound checks
    ca = math.prod(_count(q) for q in A_RINGS[:a])
    cb = math.prod(_count(q) for q in B_RINGS[:b])
    return Plan(a, b, A, B, ca, cb, float('nan'))


def poisson_requests(count: int, rate: float = 20.0, seed: int = 619003) -> list[Request]:
    """The served workload: Poisson arrivals; p uniform over the accepted primes in [499, 619];
    x_lo = 10^U(20, log10 3e27); span = 10^U(15, 22); x_hi = min(x_lo + span, 3e27)."""
    rng = random.Random(seed)
    t, out = 0.0, []
    for i in range(count):
        t += rng.expovariate(rate)
        lo = int(10 ** rng.uniform(20, math.log10(X_MAX)))
        span = int(10 ** rng.uniform(15, 22))
        hi = min(lo + span, X_MAX)
        out.append(Request(i, rng.choice(SERVED_PRIMES), lo, hi, t))
    return out


@dataclass
class Work:
    """One request in flight: its plan, its remaining windows and its accumulated result."""
    request: Request
    plan: Plan
    config: Config
    pending: deque = field(default_factory=deque)
    outstanding: int = 0
    remaining: float = 0.0
    positions: int = 0
    groups: list[int] = field(default_factory=list)
    chunks: list[np.ndarray] = field(default_factory=list)   # output records (x limb 0, x limb 1)
    windows: int = 0
    admitted: float = 0.0
    reserved: int = 0
    control: Future | None = None    # the device genuine-cube count of the request


def request_windows(req: Request, plan: Plan) -> list[tuple[Window, float]]:
    """Cut a request into windows (with their modelled positions): x sub-ranges so that one v
    row's u range stays within half a window's u budget, then v ranges within the budgets."""
    span = req.hi - req.lo
    da, db = plan.density_a, plan.density_b
    x_step = max(1, int(U_WINDOW * plan.B / (2 * da))) if da * span / plan.B > U_WINDOW / 2 else span
    out = []
    for x0 in range(req.lo, req.hi, x_step):
        x1 = min(x0 + x_step, req.hi)
        s = x1 - x0
        per_v_u = da * s / plan.B
        dv_u = (U_WINDOW / max(da, 1e-300) - s / plan.B) * plan.B / plan.A
        dv = min(dv_u, V_WINDOW / db, P_WINDOW / max(db * per_v_u, 1e-300))
        dv = max(1, int(dv))
        for v0 in range(0, plan.B, dv):
            v1 = min(v0 + dv, plan.B)
            out.append((Window(req.p, v0, v1, x0, x1, plan.A, plan.B), (v1 - v0) * db * per_v_u))
    return out


M64 = (1 << 64) - 1


def _residues(lo: np.ndarray, hi: np.ndarray, q: int) -> np.ndarray:
    """x mod q for x = hi 2^64 + lo (hi < 2^32), exactly, in uint64 arithmetic."""
    return ((hi % np.uint64(q)) * np.uint64((1 << 64) % q) + lo % np.uint64(q)) % np.uint64(q)


def _cube_mask(lo: np.ndarray, hi: np.ndarray) -> np.ndarray:
    """x is a perfect cube, exactly: the floor cube root (icbrt_many) cubed in 128-bit limbs."""
    h, l = cube_limbs(icbrt_many(lo, hi))
    return (h == hi) & (l == lo)


def verify_outputs(records: np.ndarray, lo: int, hi: int, p: int) -> tuple[list[int], int, list[dict[str, Any]]]:
    """Host re-check of every emitted value of a request (pseudocube/batch_experiment.py:138-144),
    vectorised: lo < x <= hi, no duplicates, x = +-1 mod 9, x coprime to every prime <= p and a
    cubic residue mod every q = 1 mod 3 (local3), perfect cubes separated exactly, and the standalone
    witness verifier on every non-cube.  Returns the sorted values, the cube count and the witnesses."""
    from .predicate import primes_upto, validate_p
    validate_p(p)
    if not len(records):
        return [], 0, []
    xl, xh = records[:, 0].copy(), records[:, 1] & np.uint64(0xFFFFFFFF)
    order = np.lexsort((xl, xh))
    xl, xh = xl[order], xh[order]
    if len(xl) > 1 and np.any((xl[1:] == xl[:-1]) & (xh[1:] == xh[:-1])):
        raise ArithmeticError('duplicate canonical output')
    first, last = int(xh[0]) << 64 | int(xl[0]), int(xh[-1]) << 64 | int(xl[-1])
    if not lo < first or not last <= hi:
        raise ArithmeticError('GPU/CPU disagreement: value outside the interval')
    ok = np.isin(_residues(xl, xh, 9), np.array([1, 8], dtype=np.uint64))
    for q in primes_upto(p):
        if q == 3:
            continue
        table = np.zeros(q, dtype=bool)
        table[list(allowed(q))] = True
        ok &= table[_residues(xl, xh, q).astype(np.int64)]
    if not ok.all():
        raise ArithmeticError('GPU/CPU disagreement: local test failed')
    values = [h << 64 | l for h, l in zip(xh.tolist(), xl.tolist())]
    if len(values) >= VECTOR_MIN:                        # the standalone verifier, column-wise
        _, cubes, witnesses = verify_many(xl, xh, p)
        if not witnesses.all_valid:
            raise ArithmeticError('independent witness verification failed')
        return values, int(cubes.sum()), list(witnesses) if len(witnesses) <= MATERIALISE_MAX else witnesses
    cubes = _cube_mask(xl, xh)
    hits = [verify(n, p) for n, c in zip(values, cubes.tolist()) if not c]
    if any(not h['valid_pseudocube'] for h in hits):
        raise ArithmeticError('independent witness verification failed')
    return values, int(cubes.sum()), hits


def _digest_values(values: list[int]) -> str:
    """digest() of the decimal strings of ascending values, formatted in one pass."""
    import hashlib
    return hashlib.sha256(('[' + ','.join('"%d"' % n for n in values) + ']\n').encode()).hexdigest()


def _finish(work: Work) -> dict[str, Any]:
    """Host verification and the result record of a completed request."""
    c, req = work.config, work.request
    records = np.concatenate(work.chunks) if work.chunks else np.zeros((0, 2), dtype=np.uint64)
    values, ncubes, hits = verify_outputs(records, req.lo, req.hi, req.p)
    return dict(id=req.id, p=req.p, lo=str(req.lo), hi=str(req.hi), A=str(c.A), B=str(c.B),
                focus_split=[work.plan.a, work.plan.b], filter_groups=c.filter_groups(),
                valid_focused_candidates=work.positions, group_survivors=list(work.groups),
                local_survivors=len(values), genuine_cubes=ncubes, cpu_confirmed_hits=hits,
                output_sha256=_digest_values(values), values=values, windows=work.windows)


class ServedLoop:
    """Continuous batching of range-certification requests on one device."""

    def __init__(self, runtime: Runtime, memory_cap: int = 8 << 30, tuning: dict[str, int] | None = None,
                 output_cap: int = 1 << 20) -> None:
        self.runtime, self.engine = runtime, BatchedEngine(runtime)
        self.memory_cap, self.tuning, self.output_cap = memory_cap, tuning, output_cap
        self.steps: list[dict[str, Any]] = []
        self.step_working = 8 * STEP_U + 48 * STEP_V + 32 * output_cap + (256 << 20)
        self.reserved = 0

    def _reserve(self, plan: Plan) -> int:
        """Device bytes a request holds while admitted: its focus tables (when not yet resident)
        and an output buffer share."""
        tables = 0
        for modulus, count in ((plan.A, plan.count_a), (plan.B, plan.count_b)):
            tables += min(256 << 20, 8 * count + (1 << 20))
        return tables + (16 << 20)

    def _control(self, req: Request) -> int:
        """The genuine cubes (x_lo, x_hi] must hold at bound p, counted on the device."""
        return genuine_cube_count(self.runtime, req.p, req.lo, req.hi)

    def _device_step(self, windows: list[Window]) -> tuple[np.ndarray, np.ndarray, dict[str, Any], list[int]]:
        """One multi-window launch (one subtile per window).  A step whose outputs overflow the
        output buffer is split in halves and rerun; counters of an overflowed run are complete, but
        its outputs are not, so nothing of it is kept."""
        before = self.runtime.copies()
        batch = self.engine.plan(windows, None, self.tuning, self.output_cap)
        try:
            stats = dict(batch.run())
            after = self.runtime.copies()
            stats.update(h2d_bytes=after[0] - before[0], d2h_bytes=after[1] - before[1])
            stats.update(u_entries=batch.layout['u_entries'], v_entries=batch.layout['v_entries'])
            counts, _, records = batch.raw()
            ngs = [batch.families[batch._family_of[i]].ng for i in range(len(windows))]
            return counts, records, stats, ngs
        except OverflowError:
            if len(windows) < 2:
                raise
        finally:
            batch.close()
        half = len(windows) // 2
        c1, r1, s1, n1 = self._device_step(windows[:half])
        c2, r2, s2, n2 = self._device_step(windows[half:])
        width = max(c1.shape[1], c2.shape[1])
        pad = lambda c: np.pad(c, ((0, 0), (0, width - c.shape[1])))
        r2 = r2.copy()
        if len(r2):
            tile = (r2[:, 1] >> np.uint64(32)) + np.uint64(half)
            r2[:, 1] = (r2[:, 1] & np.uint64(0xFFFFFFFF)) | (tile << np.uint64(32))
        stats = {k: s1.get(k, 0) + s2.get(k, 0) for k in ('kernel_ms', 'total_ms', 'window_ms', 'bounds_ms',
                                                        'u_entries', 'v_entries', 'launches', 'h2d_bytes', 'd2h_bytes')}
        return np.vstack([pad(c1), pad(c2)]), np.vstack([r1, r2]), stats, n1 + n2

    def run(self, requests: list[Request], realtime: bool = True, time_limit: float = float('inf'),
            splits: dict[int, tuple[int, int]] | None = None) -> dict[str, Any]:
        """Serve ``requests`` (arrival offsets in seconds from the start) and return per-request results
        with latencies (completion - arrival), plus throughput.  ``realtime=False`` releases every
        request at once; ``splits`` forces the focus split of the given request ids."""
        splits = splits or {}
        start = time.perf_counter()
        clock = (lambda: time.perf_counter() - start) if realtime else (lambda: float('inf'))
        arrivals = deque(sorted(requests, key=lambda r: r.arrival))
        waiting: deque[tuple[Request, Plan]] = deque()
        active: list[Work] = []
        results: dict[int, dict[str, Any]] = {}
        positions_total = 0
        pool = ThreadPoolExecutor(1)
        inflight: tuple[Future, list[tuple[Work, Window]]] | None = None

        def admit() -> None:
            now = clock()
            while arrivals and arrivals[0].arrival <= now:
                r = arrivals.popleft()
                forced = splits.get(r.id)
                waiting.append((r, split_plan(r.p, r.lo, r.hi, *forced) if forced else plan_request(r.p, r.lo, r.hi)))
            while waiting:
                r, plan = waiting[0]
                need = self._reserve(plan)
                if active and self.reserved + need + self.step_working > self.memory_cap:
                    break
                waiting.popleft()
                w = Work(r, plan, Config(r.p, r.lo, r.hi, plan.A, plan.B))
                w.pending.extend(request_windows(r, plan))
                w.remaining = sum(p for _, p in w.pending)
                w.groups = [0] * len(w.config.filter_groups())
                w.admitted, w.reserved = clock(), need
                # the genuine-cube control runs on the device thread ahead of the request's steps
                w.control = pool.submit(self._control, r)
                self.reserved += need
                active.append(w)

        def compose() -> list[tuple[Work, Window]]:
            chosen: list[tuple[Work, Window]] = []
            budget_p = budget_u = budget_v = 0.0
            for w in sorted((w for w in active if w.pending), key=lambda w: (w.remaining, w.request.arrival)):
                while w.pending and len(chosen) < STEP_WINDOWS:
                    win, est = w.pending[0]
                    est_u = w.plan.density_a * ((win.end - win.first) * w.plan.A / w.plan.B + (win.hi - win.lo) / w.plan.B)
                    est_v = w.plan.density_b * (win.end - win.first)
                    if chosen and (budget_p + est > STEP_P or budget_u + est_u > STEP_U or budget_v + est_v > STEP_V):
                        return chosen
                    w.pending.popleft()
                    w.outstanding += 1
                    w.remaining -= est
                    budget_p, budget_u, budget_v = budget_p + est, budget_u + est_u, budget_v + est_v
                    chosen.append((w, win))
            return chosen

        def absorb(step: list[tuple[Work, Window]], outcome: tuple) -> list[Work]:
            nonlocal positions_total
            counts, records, stats, ngs = outcome
            tiles = (records[:, 1] >> np.uint64(32)).astype(np.int64) if len(records) else np.zeros(0, np.int64)
            order = np.argsort(tiles, kind='stable')
            records, tiles = records[order], tiles[order]
            cuts = np.searchsorted(tiles, np.arange(len(step) + 1))
            for i, (w, win) in enumerate(step):
                ng = ngs[i]
                row = counts[i]
                if int(row[ng + 2]):
                    raise ArithmeticError('unsigned underflow flagged')
                w.positions += int(row[0])
                positions_total += int(row[0])
                for g in range(ng):
                    w.groups[g] += int(row[1 + g])
                got = records[cuts[i]:cuts[i + 1]]
                if len(got) != int(row[ng + 1]):
                    raise ArithmeticError('device output count disagrees with its records')
                if len(got):
                    w.chunks.append(got)
                w.windows += 1
                w.outstanding -= 1
            self.steps.append(dict(windows=len(step), positions=int(counts[:, 0].sum()),
                                   **{k: stats.get(k, 0) for k in ('kernel_ms', 'total_ms', 'window_ms', 'bounds_ms',
                                                                   'u_entries', 'v_entries', 'launches', 'h2d_bytes',
                                                                   'd2h_bytes')}))
            done = [w for w in active if not w.pending and not w.outstanding]
            for w in done:                                # their memory is free for the next admission
                active.remove(w)
                self.reserved -= w.reserved
            return done

        def finish(done: list[Work]) -> None:
            """Host verification and results of the requests a step completed."""
            for w in done:
                res = _finish(w)
                res['cube_control'] = w.control.result()
                if res['cube_control'] != res['genuine_cubes']:
                    raise ArithmeticError(f'request {w.request.id}: {res["genuine_cubes"]} genuine cubes emitted, '
                                          f'the device control counts {res["cube_control"]}')
                res['arrival'] = w.request.arrival
                res['latency'] = clock() - w.request.arrival if realtime else None
                results[w.request.id] = res

        try:
            while arrivals or waiting or active or inflight:
                if clock() > time_limit:
                    break
                admit()
                step = compose()
                if inflight:
                    fut, prev = inflight
                    outcome = fut.result()
                    inflight = None
                    if step:
                        inflight = (pool.submit(self._device_step, [w for _, w in step]), step)
                        step = []
                    done = absorb(prev, outcome)
                    if not inflight:
                        # nothing queued on the device: refill it before the host verifies the
                        # requests this step completed
                        admit()
                        step = compose()
                        if step:
                            inflight = (pool.submit(self._device_step, [w for _, w in step]), step)
                            step = []
                    finish(done)
                if step:
                    inflight = (pool.submit(self._device_step, [w for _, w in step]), step)
                elif not inflight and arrivals and not active and not waiting:
                    time.sleep(max(0.0, min(0.05, arrivals[0].arrival - clock())))
        finally:
            if inflight:
                try:
                    inflight[0].result()
                except Exception:
                    pass
            pool.shutdown(wait=True)
        elapsed = time.perf_counter() - start
        return dict(results=results, seconds=elapsed, positions=positions_total, steps=len(self.steps),
                    unfinished=[r.id for r in requests if r.id not in results])


def plain_tile_width(plan: Plan, win: Window, pair_limit: int) -> int:
    """Largest v span whose expected u count times v count stays under the plain matcher's pair
    limit: dA (dv A/B + S/B) dB dv <= limit, solved for dv."""
    da, db = plan.density_a, plan.density_b
    alpha = da * db * plan.A / plan.B
    beta = da * db * (win.hi - win.lo) / plan.B
    dv = (-beta + math.sqrt(beta * beta + 4 * alpha * pair_limit)) / (2 * alpha)
    return max(1, int(dv * 0.5))


def plain_request(runtime: Runtime, engine: BatchedEngine, req: Request, pair_limit: int = 40_000_000,
                  split: tuple[int, int] | None = None, deadline: float = float('inf')) -> dict[str, Any]:
    """One request through the plain per-tile matcher (the reference's Matcher.tile and its
    bounded pair-opportunity limit), windows as the served loop cuts them, one tile at a time."""
    plan = split_plan(req.p, req.lo, req.hi, *split) if split else plan_request(req.p, req.lo, req.hi)
    c0 = Config(req.p, req.lo, req.hi, plan.A, plan.B)
    positions, groups, values = 0, [0] * len(c0.filter_groups()), []
    matchers: dict[tuple[int, int], Matcher] = {}
    for win, _ in request_windows(req, plan):
        c = engine.config(win)
        matcher = matchers.get((win.lo, win.hi)) or matchers.setdefault((win.lo, win.hi), Matcher(runtime, c))
        af, bf = engine.focus_pair(c)
        step = plain_tile_width(plan, win, pair_limit)
        todo = deque(Tile(v, min(v + step, win.end)) for v in range(win.first, win.end, step))
        while todo:
            if time.perf_counter() > deadline:
                raise TimeoutError('plain request passed its deadline')
            tile = todo.popleft()
            try:
                row = matcher.tile(tile, af, bf, cap=1 << 31, output_cap=1 << 20)
            except OverflowError:
                if tile.end - tile.first < 2:
                    raise
                todo.extendleft(reversed(tile.split()))
                continue
            positions += row['valid_focused_candidates']
            for g, n in enumerate(row['group_survivors']):
                groups[g] += n
            values.extend(int(n) for n in row['all_values'])
    records = np.array([[n & M64, n >> 64] for n in values], dtype=np.uint64).reshape(-1, 2)
    work = Work(req, plan, c0, positions=positions, groups=groups, chunks=[records])
    return _finish(work)


def plain_loop(runtime: Runtime, requests: list[Request], time_limit: float = float('inf')) -> dict[str, Any]:
    """The sequential plain per-request loop, in arrival order and in real time."""
    engine = BatchedEngine(runtime)
    start = time.perf_counter()
    results: dict[int, dict[str, Any]] = {}
    positions = 0
    for req in sorted(requests, key=lambda r: r.arrival):
        now = time.perf_counter() - start
        if now > time_limit:
            break
        if req.arrival > now:
            time.sleep(req.arrival - now)
        try:
            res = plain_request(runtime, engine, req, deadline=start + time_limit)
        except TimeoutError:
            break
        res['arrival'] = req.arrival
        res['latency'] = time.perf_counter() - start - req.arrival
        positions += res['valid_focused_candidates']
        results[req.id] = res
    return dict(results=results, seconds=time.perf_counter() - start, positions=positions,
                unfinished=[r.id for r in requests if r.id not in results])


def latency_summary(run: dict[str, Any], requests: list[Request]) -> dict[str, Any]:
    """p50/p99 over all requests; an unfinished request counts with the run's end as its latency,
    so with any unfinished request (``censored``) the percentiles are lower bounds."""
    lat = [r['latency'] for r in run['results'].values()]
    unfinished = set(run['unfinished'])
    lat += [run['seconds'] - req.arrival for req in requests if req.id in unfinished]
    lat.sort()
    pick = lambda q: lat[min(len(lat) - 1, int(q * len(lat)))] if lat else None
    return dict(p50=pick(0.5), p99=pick(0.99), requests=len(requests), completed=len(run['results']),
                censored=bool(unfinished),
                positions_per_second=run['positions'] / run['seconds'] if run['seconds'] else None)


def rescaled(requests: list[Request], rate: float) -> list[Request]:
    """The same requests with their arrival gaps scaled to a mean rate of ``rate`` per second."""
    if not requests:
        return []
    mean_gap = requests[-1].arrival / max(1, len(requests) - 1) if len(requests) > 1 else 1.0 / rate
    scale = (1.0 / rate) / mean_gap if mean_gap > 0 else 1.0
    return [Request(r.id, r.p, r.lo, r.hi, r.arrival * scale) for r in requests]


__all__ = ['Request', 'Plan', 'plan_request', 'split_plan', 'poisson_requests', 'request_windows', 'ServedLoop',
           'plain_request', 'plain_loop', 'latency_summary', 'rescaled', 'A_RINGS', 'B_RINGS', 'SERVED_PRIMES']
