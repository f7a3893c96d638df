"""GPU checks of the served form: every request gives the same result alone and in the mix (and
under memory-limited admission), the same result as the sequential plain per-request loop, the
same output set under another focus split, and the genuine-cube count of an independent control."""
from __future__ import annotations

import pytest

from psuedocubes_b200.predicate import icbrt, primes_upto
from psuedocubes_b200.served import (Request, ServedLoop, latency_summary, plain_request, poisson_requests,
                                     plan_request)
from psuedocubes_b200.batched import BatchedEngine

pytestmark = pytest.mark.gpu

REQUESTS = [Request(0, 619, 10**20, 10**20 + 10**15), Request(1, 499, 5 * 10**23, 5 * 10**23 + 3 * 10**16),
            Request(2, 571, 2 * 10**27, 2 * 10**27 + 10**17), Request(3, 547, 10**20, 10**20 + 10**18),
            Request(4, 613, 123456789 * 10**18, 123456789 * 10**18 + 7 * 10**15)]
TIMING = ('latency', 'arrival', 'windows')


def strip(result: dict) -> dict:
    return {k: v for k, v in result.items() if k not in TIMING}


@pytest.fixture(scope='module')
def mixed(runtime):
    return ServedLoop(runtime).run(REQUESTS, realtime=False)


def test_each_request_is_the_same_alone_and_in_the_mix(runtime, mixed):
    assert not mixed['unfinished']
    for r in REQUESTS:
        alone = ServedLoop(runtime).run([r], realtime=False)
        assert strip(alone['results'][r.id]) == strip(mixed['results'][r.id]), r.id
    squeezed = ServedLoop(runtime, memory_cap=0).run(REQUESTS, realtime=False)   # one request admitted at a time
    for r in REQUESTS:
        assert strip(squeezed['results'][r.id]) == strip(mixed['results'][r.id]), r.id


def test_served_equals_the_plain_per_request_loop(runtime, mixed):
    engine = BatchedEngine(runtime)
    for r in (REQUESTS[0], REQUESTS[1], REQUESTS[4]):
        want = plain_request(runtime, engine, r)
        got = mixed['results'][r.id]
        for key in ('valid_focused_candidates', 'group_survivors', 'filter_groups', 'local_survivors',
                    'genuine_cubes', 'output_sha256', 'values', 'focus_split'):
            assert got[key] == want[key], (r.id, key)


def test_served_requests_match_oracle(mixed, oracle):
    """Three requests, each against the oracle's masked batch over the whole canonical domain
    [0, B') of the request's own focus split (A', B') from the planner: populations, filter groups,
    the complete sorted output and its digest."""
    for r in (REQUESTS[0], REQUESTS[1], REQUESTS[4]):
        got = mixed['results'][r.id]
        A, B = int(got['A']), int(got['B'])
        g = oracle.Geometry(r.p, r.lo, r.hi, A, B)
        fa, fb = oracle.OracleFocus(g, 'A'), oracle.OracleFocus(g, 'B')
        want = oracle.batch(g, fa, fb, 0, B, width=-(-B // 64), output_cap=1 << 16)
        for key in ('valid_focused_candidates', 'group_survivors', 'filter_groups', 'local_survivors',
                    'genuine_cubes'):
            assert got[key] == want[key], (r.id, key)
        values = sorted(int(n) for n in want['all_values'])
        assert got['values'] == values, r.id
        assert got['output_sha256'] == oracle.digest([str(n) for n in values]), r.id
        assert got['valid_focused_candidates'] > 10**9


def test_output_set_does_not_depend_on_the_focus_split(runtime, mixed):
    r = REQUESTS[0]
    plan = plan_request(r.p, r.lo, r.hi)
    for split in ((plan.a, plan.b + 1), (plan.a + 1, plan.b)):
        other = ServedLoop(runtime).run([r], realtime=False, splits={r.id: split})['results'][r.id]
        assert other['focus_split'] == list(split)
        assert other['values'] == mixed['results'][r.id]['values']
        assert other['genuine_cubes'] == mixed['results'][r.id]['genuine_cubes']
        assert other['valid_focused_candidates'] != mixed['results'][r.id]['valid_focused_candidates']


def test_genuine_cubes_match_an_independent_count(mixed):
    """Cubes a^3 in (lo, hi] with a coprime to every prime <= p are exactly the genuine cubes the
    sieve must emit (a cube of such a is +-1 mod 9 and a cubic residue everywhere)."""
    for r in (REQUESTS[0], REQUESTS[3]):
        ps = primes_upto(r.p)
        a = icbrt(r.lo) + 1
        count = 0
        while a ** 3 <= r.hi:
            count += all(a % q for q in ps)
            a += 1
        assert mixed['results'][r.id]['genuine_cubes'] == count
    assert mixed['results'][3]['genuine_cubes'] > 100


def test_realtime_stream_reports_latencies(runtime):
    stream = [r for r in poisson_requests(60, rate=20.0, seed=21) if r.hi - r.lo <= 10**18][:12]
    run = ServedLoop(runtime).run(stream)
    assert not run['unfinished']
    summary = latency_summary(run, stream)
    assert summary['completed'] == len(stream) and 0 <= summary['p50'] <= summary['p99']
    assert all(res['latency'] >= 0 for res in run['results'].values())
