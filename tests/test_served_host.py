"""Host logic of the served form: the focus-split planner, the window cover of a request, the
request generator and the vectorised host re-check (no GPU)."""
from __future__ import annotations

import random

import numpy as np
import pytest

from psuedocubes_b200.focus import A619, B619, Config
from psuedocubes_b200.predicate import is_perfect_cube, local3, primes_upto
from psuedocubes_b200.served import (Request, _cube_mask, _residues, plan_request, poisson_requests,
                                     request_windows, split_plan, verify_outputs)


def test_plans_pass_the_reference_bounds():
    for r in poisson_requests(300, seed=5):
        plan = plan_request(r.p, r.lo, r.hi)
        assert plan == plan_request(r.p, r.lo, r.hi)          # deterministic
        c = Config(r.p, r.lo, r.hi, plan.A, plan.B)            # raises if a bound is violated
        assert A619 % plan.A == 0 and B619 % plan.B == 0
        assert c.focuses()[0].count == plan.count_a and c.focuses()[1].count == plan.count_b


def test_windows_cover_each_request_exactly():
    rng = random.Random(3)
    reqs = poisson_requests(40, seed=9) + [Request(99, 547, 10**20, 10**20 + 10**18)]
    for r in reqs:
        plan = plan_request(r.p, r.lo, r.hi)
        wins = [w for w, _ in request_windows(r, plan)]
        if len(wins) > 20000:
            continue
        by_x: dict[tuple[int, int], list] = {}
        for w in wins:
            assert (w.A, w.B, w.p) == (plan.A, plan.B, r.p)
            by_x.setdefault((w.lo, w.hi), []).append((w.first, w.end))
        xs = sorted(by_x)
        assert xs[0][0] == r.lo and xs[-1][1] == r.hi
        assert all(a[1] == b[0] for a, b in zip(xs, xs[1:]))
        for vs in by_x.values():
            vs.sort()
            assert vs[0][0] == 0 and vs[-1][1] == plan.B
            assert all(a[1] == b[0] and a[0] < a[1] for a, b in zip(vs, vs[1:]))
    assert rng


def test_request_stream_is_reproducible():
    a, b = poisson_requests(50), poisson_requests(50)
    assert a == b
    assert all(x.arrival < y.arrival for x, y in zip(a, a[1:]))
    assert all(10**20 <= r.lo < r.hi <= 3 * 10**27 and r.p % 3 == 1 for r in a)


def test_split_plan_rejects_out_of_bound_splits():
    with pytest.raises(ValueError):
        split_plan(571, 2 * 10**27, 2 * 10**27 + 10**17, 8, 5)


def _records(values):
    return np.array([[n & (2**64 - 1), n >> 64] for n in values], dtype=np.uint64).reshape(-1, 2)


def test_vectorised_recheck_matches_the_predicate():
    rng = random.Random(619)
    xs = [rng.randrange(1, 3 * 10**27) for _ in range(3000)]
    xs += [a ** 3 for a in (1, 2, 10**9 + 7, 1442249570)] + [(10**9 + 7) ** 3 + 1]
    lo = np.array([x & (2**64 - 1) for x in xs], dtype=np.uint64)
    hi = np.array([x >> 64 for x in xs], dtype=np.uint64)
    assert _cube_mask(lo, hi).tolist() == [is_perfect_cube(x) for x in xs]
    for q in (2, 5, 7, 9, 13, 619):
        assert _residues(lo, hi, q).tolist() == [x % q for x in xs]
    p = 499
    ps = primes_upto(p)
    good = [a ** 3 for a in range(4_641_589, 4_643_000) if all(a % q for q in ps)]
    assert all(local3(n, p) for n in good)
    lo_x, hi_x = 10**20, 10**20 + 10**17
    values, cubes, hits = verify_outputs(_records(list(reversed(good))), lo_x, hi_x, p)
    assert values == sorted(good) and cubes == len(good) and hits == []
    with pytest.raises(ArithmeticError):
        verify_outputs(_records(good + [good[0]]), lo_x, hi_x, p)          # duplicate
    with pytest.raises(ArithmeticError):
        verify_outputs(_records(good + [good[0] + 9]), lo_x, hi_x, p)      # fails the local test
    with pytest.raises(ArithmeticError):
        verify_outputs(_records(good), good[0], hi_x, p)                   # outside (lo, hi]


class _FakeLoop:
    """ServedLoop with the device step replaced by counters that record every window once."""

    @staticmethod
    def make(memory_cap=8 << 30):
        from psuedocubes_b200.served import ServedLoop

        class Loop(ServedLoop):
            seen: list = []

            def _device_step(self, windows):
                Loop.seen.extend(windows)
                ng = max(len(w.config().filter_groups()) for w in windows)
                counts = np.zeros((len(windows), ng + 3), dtype=np.uint64)
                for i, w in enumerate(windows):
                    counts[i, 0] = w.end - w.first
                return counts, np.zeros((0, 2), dtype=np.uint64), dict(kernel_ms=0.1, total_ms=0.2), \
                    [len(w.config().filter_groups()) for w in windows]

            def _control(self, req):
                return Loop.control

        Loop.seen, Loop.control = [], 0
        return Loop(runtime=None, memory_cap=memory_cap)


def test_scheduler_runs_every_window_once():
    reqs = [r for r in poisson_requests(80, seed=4) if len(request_windows(r, plan_request(r.p, r.lo, r.hi))) < 400][:25]
    for cap in (8 << 30, 0):
        loop = _FakeLoop.make(cap)
        run = loop.run(reqs, realtime=False)
        assert not run['unfinished'] and set(run['results']) == {r.id for r in reqs}
        expect = [w for r in reqs for w, _ in request_windows(r, plan_request(r.p, r.lo, r.hi))]
        assert sorted(type(loop).seen, key=repr) == sorted(expect, key=repr)
        for r in reqs:
            plan = plan_request(r.p, r.lo, r.hi)
            total = sum(w.end - w.first for w, _ in request_windows(r, plan))
            assert run['results'][r.id]['valid_focused_candidates'] == total
            assert run['results'][r.id]['cube_control'] == 0
        assert loop.reserved == 0
    loop = _FakeLoop.make()
    type(loop).control = 1                           # a control that disagrees with what was emitted
    with pytest.raises(ArithmeticError):
        loop.run(reqs[:1], realtime=False)


def test_window_results_equal_per_window_batch_results():
    """WindowBatch.results() reduces the counters of all windows at once; it must give, window by
    window, the fields batch_experiment.batch_result gives for the same counters and records (here
    synthetic counters and the golden lease's 82 real survivors placed in their subtiles)."""
    import types
    import numpy as np
    from conftest import golden
    from psuedocubes_b200.batch_experiment import batch_result
    from psuedocubes_b200.batched import Window, WindowBatch
    from psuedocubes_b200.focus import A619, B619, Config
    gold = golden('golden_lease.json')
    g0, g1 = int(gold['first']), int(gold['end'])
    values = [int(n) for n in gold['result']['all_values']]
    windows = [Window(619, g0, g1), Window(499, 5, 5 + 3 * 10**8 + 7), Window(613, B619 - 10**9, B619),
               Window(571, 10**15, 10**15 + 1)]
    widths = [10**8, 1 << 27, 10**8, 10**8]
    configs = [w.config() for w in windows]
    ntiles = [-(-(w.end - w.first) // wd) for w, wd in zip(windows, widths)]
    fams = {}
    for c in configs:
        groups = c.filter_groups()
        fams.setdefault(c.p, types.SimpleNamespace(ng=len(groups), filter_groups=groups))
    families = list(fams.values())
    b = object.__new__(WindowBatch)
    b.windows, b.configs, b.widths = windows, configs, widths
    b.families = families
    b._family_of = [families.index(fams[c.p]) for c in configs]
    b.tile_base = np.array([0, *np.cumsum(ntiles)], dtype=np.uint32)
    b.ntiles = int(sum(ntiles))
    b.stride = max(f.ng for f in families) + 3
    b.sizes = np.array([x for k in range(len(windows)) for x in (1000 + k, 2000 + k)], dtype=np.uint64)
    rng = np.random.default_rng(5)
    counts = np.zeros((b.ntiles, b.stride), dtype=np.uint64)
    counts[:, :b.stride - 2] = rng.integers(0, 10**9, size=(b.ntiles, b.stride - 2), dtype=np.uint64)
    records = []
    for n in values:                                      # the golden values, in window 0's subtiles
        t = (configs[0].canonical(n)[1] - g0) // widths[0]
        records.append((n & (2**64 - 1), n >> 64 | t << 32))
    records = np.array(records, dtype=np.uint64)[rng.permutation(len(values))]
    tile_ng = np.repeat([families[f].ng for f in b._family_of], ntiles)
    counts[np.arange(b.ntiles), tile_ng + 1] = 0
    counts[np.arange(b.ntiles), tile_ng + 2] = 0
    np.add.at(counts, (records[:, 1] >> np.uint64(32)).astype(np.int64), 0)
    for t in (records[:, 1] >> np.uint64(32)).astype(np.int64):
        counts[t, tile_ng[t] + 1] += 1
    geometry = rng.integers(0, 10**6, size=(b.ntiles, 2), dtype=np.uint64)
    b.raw = lambda: (counts, geometry, records)
    rows = b.results()
    for i, (w, c) in enumerate(zip(windows, configs)):
        t0, t1 = int(b.tile_base[i]), int(b.tile_base[i + 1])
        ng = families[b._family_of[i]].ng
        tiles = (records[:, 1] >> np.uint64(32)).astype(np.int64)
        per_tile = [sorted(int(records[k, 0]) | int(records[k, 1] & np.uint64(0xFFFFFFFF)) << 64
                           for k in np.nonzero(tiles == t)[0]) for t in range(t0, t1)]
        ranges = [(v, min(v + widths[i], w.end), 0, 0) for v in range(w.first, w.end, widths[i])]
        want = batch_result(c, ranges, counts[t0:t1, :ng + 3], per_tile, [(int(a), int(b_)) for a, b_ in geometry[t0:t1]],
                            families[b._family_of[i]].filter_groups, 1 << 62)
        want.update(p=w.p, first=str(w.first), end=str(w.end), focus_u=1000 + i, focus_v=2000 + i)
        assert rows[i] == want, i
    assert rows[0]['local_survivors'] == 82 and len(rows[0]['cpu_confirmed_hits']) == 1
