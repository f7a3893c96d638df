"""GPU parity: the sm_100a path through the C ABI against the oracle and the reference's fixtures.

Order of the checks follows the reference's own GPU qualification: limb self-test, focus windows,
complete small sets, production-geometry batches, the golden lease, high-magnitude canaries,
forced overflow, plain/masked agreement.
"""
from __future__ import annotations

import hashlib
import random

import numpy as np
import pytest

from conftest import golden
from psuedocubes_b200 import _native as N
from psuedocubes_b200.batch_experiment import FusedMatcher, MaskedMatcher, compare, prepare, prepare_arrays
from psuedocubes_b200.focus import A619, B619, Config, Tile, targeted_coordinates
from psuedocubes_b200.gpu import DeviceArray, GPUFocus, Matcher
from psuedocubes_b200.optimized import BATCH_WIDTH, compute_lease, compute_leases
from psuedocubes_b200.run_production import compute_batch

pytestmark = pytest.mark.gpu

SCOPE_KEYS = ('focus_u', 'focus_v', 'cartesian_opportunities', 'valid_focused_candidates', 'genuine_cubes',
              'local_survivors', 'cube_checks', 'subtile_scopes', 'filter_groups', 'group_survivors',
              'all_values', 'cpu_confirmed_hits')


def small_config(p: int, lo: int = 0, hi: int = 100000) -> Config:
    return Config(p, lo, hi, 14 * (19 if p >= 19 else 1), 9 * (13 if p >= 13 else 1) * (31 if p >= 31 else 1))


def test_wide_limb_selftest(runtime):
    fx = golden('wide.json')
    rand = random.Random(fx['seed'])
    cases = [tuple(int(x) for x in c) for c in fx['edge']]
    cases += [tuple(rand.getrandbits(64) for _ in range(4)) for _ in range(fx['random'])]
    data = np.array(cases, dtype=np.uint64)
    out = np.zeros(3 * len(cases), dtype=np.uint64)
    runtime.call(runtime.lib.pc_selftest_wide(runtime.ctx, data.reshape(-1), out, len(cases)))
    h = hashlib.sha256()
    for (a, b, c, d), row in zip(cases, out.reshape(-1, 3)):
        diff = (a * b - c * d) % (1 << 128)
        assert (int(row[0]), int(row[1]), int(row[2])) == (diff & (2**64 - 1), diff >> 64, int(a * b < c * d))
        h.update(f'{int(row[0])},{int(row[1])},{int(row[2])};'.encode())
    assert h.hexdigest() == fx['sha256']


def test_windows_match_reference_producer(focuses619):
    fa, fb = focuses619
    for w in golden('windows.json'):
        if w['focus'] not in ('A', 'B'):
            continue
        focus = fa if w['focus'] == 'A' else fb
        values = focus.window(int(w['low']), int(w['high']), cap=1 << 30).get()
        assert len(values) == w['count']
        assert hashlib.sha256(values.tobytes()).hexdigest() == w['sha256']
        assert [str(x) for x in values[:5]] == w['head']


def test_small_focus_windows_match_reference(runtime):
    c = small_config(31)
    af, bf = c.focuses()
    gaf, gbf = GPUFocus(runtime, af), GPUFocus(runtime, bf)
    for w in golden('windows.json'):
        if not w['focus'].startswith('small31'):
            continue
        focus = gaf if w['focus'].endswith('A') else gbf
        values = focus.window(int(w['low']), int(w['high'])).get()
        assert len(values) == w['count']
        assert hashlib.sha256(values.tobytes()).hexdigest() == w['sha256']
        assert [str(x) for x in values[:400]] == w['values']


def test_random_windows_match_oracle(focuses619, oracle619, runtime):
    g, ofa, ofb = oracle619
    fa, fb = focuses619
    rng = random.Random(619003)
    for _ in range(24):
        which = rng.random() < 0.5
        gpu, orc, M = (fa, ofa, A619) if which else (fb, ofb, B619)
        span = int(10 ** rng.uniform(0, 10.5))
        low = rng.randrange(0, 2 * M - span) if which else rng.randrange(0, M - span)
        got = gpu.window(low, low + span, cap=1 << 30).get()
        want = orc.window(low, low + span, cap=1 << 30)
        assert np.array_equal(got, want), (which, low, span)
    assert fa.window(7, 7).size == 0
    with pytest.raises(OverflowError):
        fa.window(0, 10**12, cap=10)


def test_window_period_limit(runtime):
    c = small_config(7)
    af, _ = c.focuses()
    gaf = GPUFocus(runtime, af)
    with pytest.raises(OverflowError):
        gaf.window(0, af.modulus * 5000)
    values = gaf.window(0, af.modulus * 4096).get()
    assert len(values) == af.count * 4096


@pytest.mark.parametrize('p', [7, 13, 19, 31])
def test_complete_small_sets(runtime, oracle, p):
    case = next(c for c in golden('small_sets.json') if c['p'] == p)
    c = small_config(p)
    af, bf = (GPUFocus(runtime, f) for f in c.focuses())
    width = -(-c.B // 64)
    batch = prepare(runtime, c, af, bf, 0, c.B, width)
    got = MaskedMatcher(runtime, c).run(batch, output_cap=8192)
    values = sorted(int(n) for n in got['all_values'])
    assert len(values) == case['count']
    assert oracle.digest([str(n) for n in values]) == case['values_sha256']
    g = oracle.Geometry(p, c.lo, c.hi, c.A, c.B)
    want = oracle.batch(g, oracle.OracleFocus(g, 'A'), oracle.OracleFocus(g, 'B'), 0, c.B, width=width)
    for key in SCOPE_KEYS:
        assert got[key] == want[key], key


@pytest.mark.parametrize('first', [0, 246112000000000, B619 // 2, B619 - 6_400_000_000, 575222931200000000])
def test_production_batches_match_oracle(runtime, p619, focuses619, oracle, oracle619, first):
    fa, fb = focuses619
    g, ofa, ofb = oracle619
    end = min(B619, first + BATCH_WIDTH)
    batch = prepare(runtime, p619, fa, fb, first, end)
    want = oracle.batch(g, ofa, ofb, first, end)
    got = MaskedMatcher(runtime, p619).run(batch)
    for key in SCOPE_KEYS:
        assert got[key] == want[key], key


def test_every_tuning_gives_identical_batches(runtime, p619, focuses619):
    fa, fb = focuses619
    batch = prepare(runtime, p619, fa, fb, 0, BATCH_WIDTH)
    base = FusedMatcher(runtime, p619).run(batch)
    for nb in (4, 5, 6, 7, 8):
        for K in (16, 32, 64):
            for chunk in (0, 97):
                got = MaskedMatcher(runtime, p619, dict(bitset_filters=nb, block_words=K, v_chunk=chunk)).run(batch)
                compare(base, got)
                assert got['subtile_scopes'] == base['subtile_scopes']
    for threads in (512, 768, 896, 1024):
        got = MaskedMatcher(runtime, p619, dict(bitset_filters=7, block_words=32, threads=threads)).run(batch)
        compare(base, got)
        assert got['subtile_scopes'] == base['subtile_scopes']


def test_golden_lease(runtime, p619, focuses619):
    fa, fb = focuses619
    gold = golden('golden_lease.json')
    result = compute_lease(MaskedMatcher(runtime, p619), fa, fb, int(gold['first']), int(gold['end']))
    for key, value in gold['result'].items():
        assert result[key] == value, key
    assert result['subtile_scopes'][0]['transcript_sha256'] == gold['transcript_sha256']
    assert result['subtile_scopes'][0]['output_sha256'] == gold['output_sha256']
    # the receipt the ledger tests commit through the reference's ledger is this one
    strip = lambda r: {k: v for k, v in r.items() if not k.endswith('_seconds')}
    assert strip(result) == strip(golden('golden_lease_receipt.json')['receipt'])


def test_lease_path_equals_batch_path(runtime, p619, focuses619):
    fa, fb = focuses619
    first, end = 658625401600000000, 658625401600000000 + 3 * BATCH_WIDTH + 12345
    matcher = MaskedMatcher(runtime, p619)
    fused = compute_lease(matcher, fa, fb, first, end)

    class PerBatch:
        def __init__(self, inner):
            self.inner, self.runtime, self.config = inner, inner.runtime, inner.config

        def run(self, batch):
            return self.inner.run(batch)

    batchwise = compute_lease(PerBatch(matcher), fa, fb, first, end)
    strip = lambda r: {k: v for k, v in r.items() if not k.endswith('_seconds')}
    assert strip(fused) == strip(batchwise)


def test_overlapped_leases_equal_one_by_one(runtime, p619, focuses619):
    """compute_leases overlaps the device call of the next lease with the receipt of the current
    one; every receipt must equal compute_lease of the same lease, in the given order."""
    fa, fb = focuses619
    gold = golden('golden_lease.json')
    g0 = int(gold['first'])
    leases = [(g0, int(gold['end'])), (658625401600000000, 658625401600000000 + 2 * BATCH_WIDTH + 777),
              (12345, 12345 + BATCH_WIDTH)]
    matcher = MaskedMatcher(runtime, p619)
    strip = lambda r: {k: v for k, v in r.items() if not k.endswith('_seconds')}
    got = [strip(r) for r in compute_leases(matcher, fa, fb, leases)]
    want = [strip(compute_lease(matcher, fa, fb, first, end)) for first, end in leases]
    assert got == want
    assert got[0]['subtile_scopes'][0]['transcript_sha256'] == gold['transcript_sha256']
    # two chunks through the same buffers, and a lease whose outputs overflow the list's buffer
    # (rerun alone under the reference's overflow rule)
    assert [strip(r) for r in compute_leases(matcher, fa, fb, leases[::-1] + leases, chunk=2)] == want[::-1] + want
    small = MaskedMatcher(runtime, p619)
    small.lease_output_records = 16                  # the golden lease emits 82 values
    assert [strip(r) for r in compute_leases(small, fa, fb, leases, chunk=2)] == want
    with pytest.raises(ValueError):
        list(compute_leases(matcher, fa, fb, [(10, 10)]))


def test_overlapped_leases_stopped_early(runtime, p619, focuses619):
    """A consumer that stops after two receipts: the leases already issued finish on the helper
    thread before the generator returns, and the context is free for the next call."""
    fa, fb = focuses619
    matcher = MaskedMatcher(runtime, p619)
    leases = [(12345 + k * BATCH_WIDTH, 12345 + (k + 1) * BATCH_WIDTH) for k in range(6)]
    beats = []
    gen = compute_leases(matcher, fa, fb, leases, heartbeat=lambda: beats.append(1), chunk=2)
    got = [next(gen), next(gen)]
    gen.close()
    assert len(beats) == 2
    strip = lambda r: {k: v for k, v in r.items() if not k.endswith('_seconds')}
    assert [strip(r) for r in got] == [strip(compute_lease(matcher, fa, fb, f, e)) for f, e in leases[:2]]
    again = compute_lease(matcher, fa, fb, *leases[5])
    assert strip(again) == strip(list(compute_leases(matcher, fa, fb, leases[5:]))[0])


def test_high_magnitude_canaries(runtime, focuses619):
    """N613 at p=613 and two cubes at p=619, each alone in a narrow interval
    (tools/run_production.py:102-105)."""
    fa, fb = focuses619
    for case in golden('known.json')['cases']:
        p, n = case['p'], int(case['n'])
        narrow = Config(p, n - 1, n, A619, B619)
        v = narrow.canonical(n)[1]
        tile = Tile(max(0, v - 5_000_000), min(B619, v + 5_000_001))
        assert Matcher(runtime, narrow).tile(tile, fa, fb)['all_values'] == [str(n)]
        width = -(-(tile.end - tile.first) // 64)
        batch = prepare(runtime, narrow, fa, fb, tile.first, tile.end, width)
        assert MaskedMatcher(runtime, narrow).run(batch)['all_values'] == [str(n)]
        wide = Config(p, max(0, n - 100), min(3 * 10**27, n + 100), A619, B619)
        us, vs = targeted_coordinates(wide, n)
        assert str(n) in Matcher(runtime, wide).coordinates(us, vs)['all_values']


def test_forced_overflow_and_invalid_arguments(runtime):
    c = small_config(7)
    af, bf = (GPUFocus(runtime, f) for f in c.focuses())
    batch = prepare(runtime, c, af, bf, 0, c.B, 1)
    with pytest.raises(OverflowError):
        MaskedMatcher(runtime, c).run(batch, output_cap=1)
    with pytest.raises(ValueError):
        MaskedMatcher(runtime, c).run(batch, output_cap=0)
    m = Matcher(runtime, c)
    with pytest.raises(OverflowError):
        m.arrays(batch.us, batch.vs, cap=1)
    with pytest.raises(ValueError):
        Matcher(runtime, c, variant='unknown')


def test_plain_batch_equals_masked(runtime, p619, focuses619):
    fa, fb = focuses619
    first, end = 100_000_000, 100_000_000 + BATCH_WIDTH
    plain = compute_batch(Matcher(runtime, p619), fa, fb, first, end, 100_000_000)
    masked = MaskedMatcher(runtime, p619).run(prepare(runtime, p619, fa, fb, first, end))
    for key in ('valid_focused_candidates', 'group_survivors', 'subtile_scopes', 'all_values', 'focus_v',
                'genuine_cubes', 'local_survivors'):
        assert plain[key] == masked[key], key


@pytest.mark.parametrize('case', ['p499', 'p613', 'p571-request-split'])
def test_plain_tiles_match_oracle(runtime, focuses619, oracle, oracle619, case):
    """The plain matcher (the baseline of the batched and served forms) against the oracle's plain
    tile at prime bounds other than 619, and with a focus split the served planner chooses."""
    from psuedocubes_b200.served import plan_request
    if case == 'p571-request-split':
        lo, hi = 2 * 10**27, 2 * 10**27 + 10**17
        plan = plan_request(571, lo, hi)
        c = Config(571, lo, hi, plan.A, plan.B)
        fa, fb = (GPUFocus(runtime, f) for f in c.focuses())
        g = oracle.Geometry(571, lo, hi, plan.A, plan.B)
        ofa, ofb = oracle.OracleFocus(g, 'A'), oracle.OracleFocus(g, 'B')
        tile = Tile(plan.B // 3, plan.B // 3 + plan.B // 2000)       # within the 5e7 pair limit
    else:
        p = int(case[1:])
        c = Config(p, 10**27, 3 * 10**27, A619, B619)
        fa, fb = focuses619
        _, ofa, ofb = oracle619
        g = oracle.Geometry(p, c.lo, c.hi, A619, B619)
        tile = Tile(658625401600000000, 658625401600000000 + 100_000_000)
    got = Matcher(runtime, c).tile(tile, fa, fb, output_cap=1 << 16)
    us = ofa.window(c.u_interval(tile.first)[0], c.u_interval(tile.end - 1)[1], cap=1 << 30)
    vs = ofb.window(tile.first, tile.end, cap=1 << 30)
    want = oracle.plain_tile(g, us, vs, output_cap=1 << 16)
    ng = len(g.filter_groups)
    pops = want['populations']
    assert got['focus_u'] == len(us) and got['focus_v'] == len(vs)
    assert got['valid_focused_candidates'] == pops[0] > 0
    assert got['group_survivors'] == pops[1:ng + 1]
    assert got['local_survivors'] == pops[ng + 1] and pops[ng + 2] == 0
    assert [int(n) for n in got['all_values']] == want['values']


def test_p67_prefix(runtime, oracle):
    case = golden('p67_prefix.json')
    c = Config(67, 1, 10**13, case['A'], case['B'])
    af, bf = (GPUFocus(runtime, f) for f in c.focuses())
    end = case['v_end']
    width = -(-end // 64)
    batch = prepare(runtime, c, af, bf, 0, end, width)
    with pytest.raises(OverflowError):      # ~12.5k outputs per focus v: the 8192-per-subtile cap trips
        MaskedMatcher(runtime, c).run(batch)
    raw = MaskedMatcher(runtime, c).run_lease(af, bf, 0, end, width, output_cap=1 << 20)
    values = sorted(n for tile in raw['per_tile'] for n in tile)
    assert len(values) == case['count']
    assert oracle.digest([str(n) for n in values]) == case['values_sha256']


def test_coordinates_upload_roundtrip(runtime):
    data = np.array([1, 5, 9, 2**63 + 1], dtype=np.uint64)
    arr = DeviceArray.from_host(runtime, data)
    assert np.array_equal(arr.get(), data)
    assert np.array_equal(arr[1:3].get(), data[1:3])
    assert arr.searchsorted([0, 5, 6, 2**64 - 1]).tolist() == [0, 1, 2, 4]
    assert arr[1:3].searchsorted([0, 5, 6, 2**64 - 1]).tolist() == [0, 0, 1, 2]


@pytest.mark.parametrize('index', [0, 3, 24])
def test_bench_lease_batches_match_oracle(runtime, p619, focuses619, oracle, oracle619, index):
    """Leases bench.py times: lease 0 (its first warm-up lease), 3 (the first timed lease at its
    default --warmup 3) and 24 (the last timed lease at --warmup 5 --steps 20): the first, a middle
    and the last batch of each, subtile by subtile, against the oracle."""
    import bench
    fa, fb = focuses619
    g, ofa, ofb = oracle619
    first, end = bench.lease_bounds(index)
    raw = MaskedMatcher(runtime, p619).run_lease(fa, fb, first, end, 100_000_000)
    ng = len(p619.filter_groups())
    for b in (0, 131, 255):
        start = first + b * BATCH_WIDTH
        want = oracle.batch(g, ofa, ofb, start, start + BATCH_WIDTH)
        for k, scope in enumerate(want['subtile_scopes']):
            t = 64 * b + k
            row = raw['counts'][t]
            assert int(row[0]) == scope['valid_focused_candidates'], (b, k)
            assert [int(n) for n in row[1:ng + 1]] == scope['group_survivors'], (b, k)
            assert int(row[ng + 1]) == scope['local_survivors'] and int(row[ng + 2]) == 0
            assert oracle.digest([str(n) for n in raw['per_tile'][t]]) == scope['output_sha256']
        geo = raw['geometry'][64 * b:64 * b + 64]
        assert int(geo[:, 0].sum()) == want['focus_u'] and int(geo[:, 1].sum()) == want['focus_v']


@pytest.mark.parametrize('index', [5, 25])
def test_bench_leases_match_oracle_whole(runtime, p619, focuses619, oracle, oracle619, index):
    """At --warmup 5 --steps 20, lease 5 is the first lease bench.py times on the device and lease
    25 the first of its end-to-end run through compute_leases.  Each is checked whole against the
    oracle's lease: all 256 batches, through the transcript over 16,384 subtile scopes, the
    output hash, the populations and the values."""
    import os
    import bench
    fa, fb = focuses619
    g, ofa, ofb = oracle619
    first, end = bench.lease_bounds(index)
    got = compute_lease(MaskedMatcher(runtime, p619), fa, fb, first, end)
    workers = max(1, (os.cpu_count() or 2) // 2)
    want = oracle.lease(g, ofa, ofb, first, end, workers=workers, threads_per_batch=2)
    scope = got['subtile_scopes'][0]
    assert scope['transcript_sha256'] == want['transcript_sha256']
    assert scope['output_sha256'] == want['output_sha256']
    for key in ('focus_u', 'focus_v', 'cartesian_opportunities', 'valid_focused_candidates', 'genuine_cubes',
                'local_survivors', 'group_survivors', 'filter_groups', 'all_values', 'compute_batches',
                'subtiles_executed'):
        assert got[key] == want[key], key
    assert [h['n'] for h in got['cpu_confirmed_hits']] == [h['n'] for h in want['cpu_confirmed_hits']]


def test_calls_report_the_bytes_they_copy(runtime, p619, focuses619):
    """pc_stats counts the library's own host transfers: a lease uploads its window, segment and
    subtile descriptors and brings back counters, envelope sizes, records and scalars."""
    import ctypes
    from psuedocubes_b200.gpu import MASK
    fa, fb = focuses619
    m = MaskedMatcher(runtime, p619)
    first, end = 658625401600000000, 658625401600000000 + 2 * BATCH_WIDTH
    nt, ng = 128, len(m.filter_groups)
    counts, geometry = np.zeros(nt * (ng + 3), dtype=np.uint64), np.zeros(2 * nt, dtype=np.uint64)
    records, n_out, stats = np.zeros(2 * 1024, dtype=np.uint64), ctypes.c_uint64(), N.Stats()
    c = p619
    runtime.call(runtime.lib.pc_run_lease(runtime.ctx, fa.handle, fb.handle, m.filters.handle, ctypes.byref(m.tuning),
                                          first, end, 100_000_000, c.lo & MASK, c.lo >> 64, c.hi & MASK, c.hi >> 64,
                                          counts, geometry, records, 1024, ctypes.byref(n_out), ctypes.byref(stats)))
    s = stats.as_dict()
    assert nt * 4 <= s['h2d_bytes'] < 1 << 20                        # the subtile map and descriptors
    assert s['d2h_bytes'] >= counts.nbytes + geometry.nbytes + 16 + 16 * n_out.value
