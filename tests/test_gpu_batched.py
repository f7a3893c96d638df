"""GPU parity of the batched form: many windows with different prime bounds, foci and intervals in
one launch sequence, each checked against the oracle, against the plain per-tile path of the same
build and, where the reference holds a fixture, against it; graph replays must equal the eager
run."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden
from psuedocubes_b200.batched import WORKLOAD_PRIMES, Autotuner, BatchedEngine, Window, seeded_windows
from psuedocubes_b200.batch_experiment import MaskedMatcher
from psuedocubes_b200.focus import B619
from psuedocubes_b200.gpu import Matcher
from psuedocubes_b200.optimized import BATCH_WIDTH
from psuedocubes_b200.run_production import compute_batch

pytestmark = pytest.mark.gpu

KEYS = ('valid_focused_candidates', 'group_survivors', 'filter_groups', 'local_survivors', 'genuine_cubes')
P67 = dict(A=2523326, B=2486169, lo=1, hi=10**13)


@pytest.fixture(scope='module')
def engine(runtime):
    return BatchedEngine(runtime)


def plain(runtime, engine, w: Window, tile: int) -> dict:
    """The plain per-tile loop of the same build over the window's v range."""
    c = w.config()
    af, bf = c.focuses()
    return compute_batch(Matcher(runtime, c), engine.focus(af), engine.focus(bf), w.first, w.end, tile)


def assert_same(got: dict, want: dict) -> None:
    for key in KEYS:
        assert got[key] == want[key], key
    assert sorted(int(n) for n in got['all_values']) == sorted(int(n) for n in want['all_values'])


def test_mixed_prime_bounds_match_plain_path(runtime, engine):
    windows = [Window(619, 0, 1_000_000_000), Window(499, B619 - 3_000_000_000, B619),
               Window(571, 658625401600000000, 658625401600000000 + 2_500_000_000),
               Window(613, 575222931200000000, 575222931200000000 + BATCH_WIDTH),
               Window(547, 12345, 12346), Window(523, 10**17, 10**17 + 1_000_003)]
    batch = engine.plan(windows, width=1 << 24)
    batch.run()
    rows = batch.results()
    for w, row in zip(windows, rows):
        assert_same(row, plain(runtime, engine, w, 100_000_000))
    assert rows[3]['valid_focused_candidates'] > 10**9
    batch.close()


def test_every_workload_prime_matches_oracle(runtime, engine, oracle, oracle619):
    """24 seeded windows of the batched workload's span distribution, their prime bounds cycling
    through every p of the workload (499 ... 619), in one launch sequence: every window's
    populations, filter groups and complete sorted output against the oracle's masked batch over
    the same Geometry (the A619/B619 focus tables do not depend on p)."""
    _, ofa, ofb = oracle619
    spans = seeded_windows(24, seed=499, span_exp=(6.0, 9.7))
    windows = [Window(WORKLOAD_PRIMES[i % len(WORKLOAD_PRIMES)], w.first, w.end) for i, w in enumerate(spans)]
    batch = engine.plan(windows, width=1 << 27)
    batch.run()
    rows = batch.results()
    batch.close()
    for w, row in zip(windows, rows):
        g = oracle.Geometry(w.p, w.lo, w.hi, w.A, w.B)
        want = oracle.batch(g, ofa, ofb, w.first, w.end, width=-(-(w.end - w.first) // 64), output_cap=1 << 16)
        for key in ('valid_focused_candidates', 'group_survivors', 'filter_groups', 'local_survivors',
                    'genuine_cubes'):
            assert row[key] == want[key], (w, key)
        assert sorted(int(n) for n in row['all_values']) == sorted(int(n) for n in want['all_values']), w
    assert sum(row['valid_focused_candidates'] for row in rows) > 10**9


@pytest.mark.parametrize('width', [1, 5])
def test_fine_subtiles_match_oracle(runtime, engine, oracle, width):
    """Subtiles so narrow that one work item spans hundreds of them: a piece's further marked
    units wait on the leftover list with subtile slots past its 8-bit field, which are recomputed
    from v, and the survivor counters go to global memory past the shared slots.  At p = 31 the
    bitset filters (q = 5, 11, 17, 23, 29, none 1 mod 3) keep every position, so nearly every unit
    of a piece goes through the leftover list.  The oracle's masked batch takes at most 64
    subtiles, so it runs over consecutive 64-subtile stretches of the window; every subtile's scope
    and the window's totals are checked against them."""
    w = Window(31, 0, 3627, 0, 100000, 266, 3627)
    batch = engine.plan([w], width=width, output_cap=1 << 16)
    batch.run()
    row = batch.results()[0]
    batch.close()
    g = oracle.Geometry(w.p, w.lo, w.hi, w.A, w.B)
    fa, fb = oracle.OracleFocus(g, 'A'), oracle.OracleFocus(g, 'B')
    parts = [oracle.batch(g, fa, fb, a, min(a + 64 * width, w.end), width=width, output_cap=1 << 16)
             for a in range(w.first, w.end, 64 * width)]
    assert len(row['subtile_scopes']) == -(-w.end // width) > 255
    assert row['subtile_scopes'] == [sc for part in parts for sc in part['subtile_scopes']]
    for key in ('cartesian_opportunities', 'valid_focused_candidates', 'genuine_cubes', 'local_survivors',
                'cube_checks'):
        assert row[key] == sum(part[key] for part in parts), key
    assert row['group_survivors'] == [sum(col) for col in zip(*(part['group_survivors'] for part in parts))]
    assert row['filter_groups'] == parts[0]['filter_groups']
    assert sorted(int(n) for n in row['all_values']) == sorted(int(n) for part in parts for n in part['all_values'])
    assert row['local_survivors'] > 0


def test_subtile_width_does_not_change_window_results(runtime, engine):
    windows = seeded_windows(24, seed=7, span_exp=(6.0, 9.3))
    base = None
    for width in (1 << 20, 1 << 24, 1 << 27, 10**8):
        batch = engine.plan(windows, width=width)
        batch.run()
        rows = [{k: r[k] for k in KEYS + ('all_values', 'focus_u', 'focus_v')} for r in batch.results()]
        batch.close()
        if base is None:
            base = rows
        assert rows == base, width


def test_graph_replay_equals_eager(runtime, engine):
    windows = seeded_windows(48, seed=11, span_exp=(6.0, 9.5))
    batch = engine.plan(windows, width=1 << 22)
    batch.run()
    counts, geometry, records = batch.raw()
    eager_rows = batch.results()
    for _ in range(3):
        stats = batch.run(graph=True)
        assert stats['graph']
        c2, g2, r2 = batch.raw()
        assert np.array_equal(counts, c2) and np.array_equal(geometry, g2)
        assert sorted(map(tuple, records.tolist())) == sorted(map(tuple, r2.tolist()))
        assert batch.results() == eager_rows
    batch.close()


def test_other_foci_and_small_families_in_one_launch(runtime, engine, oracle):
    """Windows with different focus moduli (p=67 split, the p=31 small set) beside p=619 windows:
    per-segment bitset filters, cheap tier and deep filters all switch inside one launch."""
    windows = [Window(31, 0, 3627, 0, 100000, 266, 3627),
               Window(67, 0, 2000, **P67), Window(67, 2486169 - 1500, 2486169, **P67),
               Window(619, 246112000000000, 246112000000000 + 700_000_000)]
    batch = engine.plan(windows, width=1 << 20, output_cap=1 << 20)
    batch.run()
    rows = batch.results()
    case = next(c for c in golden('small_sets.json') if c['p'] == 31)
    values = sorted(int(n) for n in rows[0]['all_values'])
    assert len(values) == case['count']
    assert oracle.digest([str(n) for n in values]) == case['values_sha256']
    assert rows[0]['local_survivors'] == case['count']
    for w, row in zip(windows[1:3], rows[1:3]):
        c = w.config()
        af, bf = (engine.focus(f) for f in c.focuses())
        us = af.window(c.u_interval(w.first)[0], c.u_interval(w.end - 1)[1], cap=1 << 30)
        vs = bf.window(w.first, w.end)
        want = Matcher(runtime, c).arrays(us, vs, cap=1 << 20)
        assert_same(row, want)
    assert_same(rows[3], plain(runtime, engine, windows[3], 100_000_000))
    assert batch.layout['bitset_filters'] == 5                 # the p=31 family has five filters
    batch.close()
    with pytest.raises(ValueError):                             # one filter cannot share a bitset tier of four
        engine.plan([Window(7, 0, 9, 0, 100000, 14, 9), Window(619, 0, 10**6)])


def test_one_window_batch_equals_lease_call(runtime, engine, p619, focuses619):
    first = 658625401600000000
    end = first + 3 * BATCH_WIDTH + 12345
    fa, fb = focuses619
    lease = MaskedMatcher(runtime, p619).run_lease(fa, fb, first, end, 100_000_000, output_cap=1 << 16)
    batch = engine.plan([Window(619, first, end)], width=100_000_000)
    batch.run()
    counts, geometry, records = batch.raw()
    ng = len(p619.filter_groups())
    assert np.array_equal(counts[:, :ng + 3], lease['counts'])
    assert np.array_equal(geometry, lease['geometry'])
    assert sorted(int(a) | (int(b) & 0xFFFFFFFF) << 64 for a, b in records) == \
        sorted(n for t in lease['per_tile'] for n in t)
    tiles = sorted((int(a) | (int(b) & 0xFFFFFFFF) << 64, int(b) >> 32) for a, b in records)
    assert tiles == sorted((n, t) for t, values in enumerate(lease['per_tile']) for n in values)
    batch.close()


def test_output_overflow_and_invalid_windows(runtime, engine):
    with pytest.raises(OverflowError):
        batch = engine.plan([Window(31, 0, 3627, 0, 100000, 266, 3627)], width=1 << 20, output_cap=10)
        batch.run()
    with pytest.raises(ValueError):
        engine.plan([Window(619, 10, 10)])
    with pytest.raises(ValueError):
        engine.plan([Window(619, B619 - 5, B619 + 5)])


def test_autotuner_persists_a_choice(runtime, engine, tmp_path):
    windows = seeded_windows(16, seed=3, span_exp=(6.0, 8.5))
    tuner = Autotuner(engine, tmp_path / 'tuning.json', replays=1)
    first = tuner.tune(windows)
    assert first.trials and first.settings['deep_records'] >= 1024
    again = tuner.tune(windows)
    assert again.settings == first.settings
    batch = engine.plan(windows, first.settings['width'], {k: v for k, v in first.settings.items() if k != 'width'})
    batch.run(graph=True)
    ref = engine.plan(windows, 1 << 26)
    ref.run()
    assert [r['all_values'] for r in batch.results()] == [r['all_values'] for r in ref.results()]
    assert [r['group_survivors'] for r in batch.results()] == [r['group_survivors'] for r in ref.results()]
    batch.close()
    ref.close()


def test_stream_equals_one_set_at_a_time(runtime, engine):
    """BatchedEngine.stream overlaps the host results of one window set with the device run of
    the next; every set's results must equal planning and running it alone, in order, and a
    consumer that stops early leaves the engine usable."""
    sets = [seeded_windows(12, seed=s, span_exp=(6.0, 9.0)) for s in (1, 2, 3)]
    want = []
    for ws in sets:
        b = engine.plan(ws, width=1 << 24)
        b.run()
        want.append(b.results())
        b.close()
    assert list(engine.stream(sets, width=1 << 24)) == want
    gen = engine.stream(sets, width=1 << 24)
    assert next(gen) == want[0]
    gen.close()
    assert list(engine.stream(sets[2:], width=1 << 24, graph=True)) == want[2:]
