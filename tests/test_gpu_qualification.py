"""The reference's GPU qualification cases, run through this build's device path.

The reference qualifies a GPU deployment with a correctness suite and a full-lease equivalence
run (tools/gpu_worker.py:70-131 and tools/qualify_optimized.py:36-61 of its release archive
releases/20260916-exhaust-v1.tar.gz):

* a forced output overflow is detected, and the same work replayed with room succeeds;
* a tile whose outputs overflow is invalidated, split, and both halves replayed give the
  complete p = 7 set;
* a wrong device residue table surfaces as an integrity failure of the host re-check;
* an interval whose lower endpoint is the known value excludes it;
* a noncube built from chosen residues by the CRT is found;
* a full 256-batch lease through the masked engine equals the plain per-tile loop, and so do
  the batches at three boundary positions of the canonical domain.

Every case fails on the host or runs ordinary inputs; none can fault the device.
"""
from __future__ import annotations

from math import prod

import pytest

from conftest import golden
from psuedocubes_b200.accounting import digest
from psuedocubes_b200.batch_experiment import MaskedMatcher, compare, prepare
from psuedocubes_b200.focus import A619, B619, Config, Tile, targeted_coordinates
from psuedocubes_b200.gpu import Filters, GPUFocus, Matcher
from psuedocubes_b200.optimized import BATCH_WIDTH, LEASE_WIDTH, PROFILE, Accumulator, compute_lease
from psuedocubes_b200.run_production import compute_batch

pytestmark = pytest.mark.gpu

P7 = Config(7, 0, 100000, 14, 9)


@pytest.fixture(scope='module')
def p7_set(oracle):
    """The complete p = 7 set for x <= 10^5, from the exact predicate."""
    return {n for n in range(1, 100001) if oracle.local3(n, 7)}


def test_forced_output_overflow_is_detected_and_replayed(runtime):
    matcher = Matcher(runtime, P7)
    us, vs = targeted_coordinates(P7, 1)
    with pytest.raises(OverflowError):
        matcher.coordinates(us, vs, cap=0)
    row = matcher.coordinates(us, vs)
    assert row['status'] == 'PASS' and '1' in row['all_values']


def test_overflowing_tile_is_split_and_both_halves_replayed(runtime, p7_set):
    matcher = Matcher(runtime, P7)
    af, bf = (GPUFocus(runtime, f) for f in P7.focuses())
    whole = Tile(0, P7.B)
    with pytest.raises(OverflowError):
        matcher.tile(whole, af, bf, output_cap=0)
    replayed = []
    for child in whole.split():
        replayed.extend(int(n) for n in matcher.tile(child, af, bf)['all_values'])
    assert len(replayed) == len(set(replayed)) and set(replayed) == p7_set

    class Capped:
        """The plain matcher with an output capacity below the whole tile's 2,541 values but above
        either v row's (1,271 and 1,270), so compute_batch must split the tile once."""
        config, filter_groups = matcher.config, matcher.filter_groups

        def tile(self, tile, af, bf):
            return matcher.tile(tile, af, bf, output_cap=2000)

    split = compute_batch(Capped(), af, bf, 0, P7.B, P7.B)
    whole_row = compute_batch(matcher, af, bf, 0, P7.B, P7.B)
    assert split['overflow_splits'] and not whole_row['overflow_splits']
    assert {int(n) for n in split['all_values']} == p7_set
    for key in ('valid_focused_candidates', 'group_survivors', 'local_survivors', 'genuine_cubes'):
        assert split[key] == whole_row[key], key


def test_wrong_device_table_is_an_integrity_failure(runtime):
    config = Config(13, 0, 100000, 14, 117)
    af, bf = (GPUFocus(runtime, f) for f in config.focuses())
    us = af.window(config.u_interval(0)[0], config.u_interval(config.B - 1)[1])
    vs = bf.window(0, config.B)
    good = Matcher(runtime, config)
    assert good.arrays(us, vs, cap=1 << 20)['status'] == 'PASS'
    bad = Matcher(runtime, config)
    bad.filters = Filters(runtime, config, table=[1] * sum(config.filter_order()))   # every residue allowed
    with pytest.raises(ArithmeticError):
        bad.arrays(us, vs, cap=1 << 20)
    masked = MaskedMatcher(runtime, config)
    masked.filters = Filters(runtime, config, table=[1] * sum(config.filter_order()))
    width = -(-config.B // 64)
    with pytest.raises(ArithmeticError):
        masked.run(prepare(runtime, config, af, bf, 0, config.B, width))


def test_excluded_lower_endpoint_emits_nothing(runtime, focuses619):
    fa, fb = focuses619
    for case in golden('known.json')['cases']:
        p, n = case['p'], int(case['n'])
        excluded = Config(p, n, n + 1, A619, B619)
        v = excluded.canonical(n)[1]
        tile = Tile(max(0, v - 5_000_000), min(B619, v + 5_000_001))
        assert Matcher(runtime, excluded).tile(tile, fa, fb)['all_values'] == []
        width = -(-(tile.end - tile.first) // 64)
        batch = prepare(runtime, excluded, fa, fb, tile.first, tile.end, width)
        assert MaskedMatcher(runtime, excluded).run(batch)['all_values'] == []


def test_crt_constructed_noncube_is_found(runtime, oracle):
    moduli, residues = [2, 5, 7, 9, 11, 13], [1, 2, 1, 8, 3, 12]
    modulus = prod(moduli)
    n = sum(r * (modulus // q) * pow(modulus // q, -1, q) for q, r in zip(moduli, residues)) % modulus
    assert oracle.local3(n, 13) and not oracle.is_cube(n)
    config = Config(13, n - 1, n, 14, 117)
    us, vs = targeted_coordinates(config, n)
    row = Matcher(runtime, config).coordinates(us, vs)
    assert row['all_values'] == [str(n)] and row['cpu_confirmed_hits'] == [str(n)]


def signature(row: dict) -> str:
    """Digest of a receipt without its timings (tools/qualify_optimized.py:25-26)."""
    return digest({k: v for k, v in row.items() if not k.endswith('_seconds')})


def test_full_lease_masked_equals_plain_loop(runtime, p619, focuses619):
    fa, fb = focuses619
    plain = Matcher(runtime, p619)
    acc = Accumulator(0, LEASE_WIDTH)
    for first in range(0, LEASE_WIDTH, BATCH_WIDTH):
        acc.add(first, first + BATCH_WIDTH,
                compute_batch(plain, fa, fb, first, first + BATCH_WIDTH, PROFILE['tile_width']))
    baseline = acc.finish(0.0)
    actual = compute_lease(MaskedMatcher(runtime, p619), fa, fb, 0, LEASE_WIDTH)
    assert signature(baseline) == signature(actual)
    assert actual['valid_focused_candidates'] > 10**11


@pytest.mark.parametrize('first,end', [(246112000000000, 246112000000000 + BATCH_WIDTH),
                                       (B619 // 2, B619 // 2 + BATCH_WIDTH), (B619 - 100000001, B619)])
def test_boundary_batches_masked_equal_plain(runtime, p619, focuses619, first, end):
    fa, fb = focuses619
    old = compute_batch(Matcher(runtime, p619), fa, fb, first, end, PROFILE['tile_width'])
    new = MaskedMatcher(runtime, p619).run(prepare(runtime, p619, fa, fb, first, end, PROFILE['tile_width']))
    compare(old, new)
