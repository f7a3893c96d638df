"""The CPU oracle pinned against the reference's own golden vectors and tools.

Fixtures in tests/golden were produced by tests/golden/make_golden.py from the reference's Python,
its compiled review tools (focus_window_cpu.cpp, wide.c) and its golden lease replay.
"""
from __future__ import annotations

import hashlib
import os
import random

import numpy as np
import pytest

from conftest import golden


def test_golden_lease_bit_exact(oracle, oracle619):
    """All 256 batches of the reference's golden lease: counts, 24 group populations, the 82 values
    in order, the witness, the transcript and the output hash."""
    g, fa, fb = oracle619
    gold = golden('golden_lease.json')
    r = oracle.lease(g, fa, fb, int(gold['first']), int(gold['end']), workers=8, threads_per_batch=1)
    for key in ('focus_u', 'focus_v', 'cartesian_opportunities', 'valid_focused_candidates', 'genuine_cubes',
                'local_survivors', 'cube_checks', 'group_survivors', 'filter_groups', 'all_values',
                'cpu_confirmed_hits', 'compute_batches', 'subtiles_executed'):
        assert r[key] == gold['result'][key], key
    assert r['transcript_sha256'] == gold['transcript_sha256']
    assert r['output_sha256'] == gold['output_sha256']


def test_batch_zero_known_populations(oracle, oracle619):
    g, fa, fb = oracle619
    r = oracle.batch(g, fa, fb, 0, 6_400_000_000)
    assert (r['focus_u'], r['focus_v'], r['cartesian_opportunities'], r['valid_focused_candidates']) == \
        (1143275, 61762, 1103295382, 1065957260)
    assert r['group_survivors'][:5] == [12908557, 157052, 1894, 29, 0]
    assert r['all_values'] == []


def test_windows_match_reference_producer(oracle, oracle619):
    """Windows of the p=619 focuses equal the reference's focus_window_cpu.cpp output."""
    g, fa, fb = oracle619
    for w in golden('windows.json'):
        if w['focus'] not in ('A', 'B'):
            continue
        focus = fa if w['focus'] == 'A' else fb
        values = focus.window(int(w['low']), int(w['high']), cap=1 << 30)
        assert len(values) == w['count']
        assert hashlib.sha256(values.tobytes()).hexdigest() == w['sha256']


def test_small_sets_match_enumerate_cpu(oracle):
    """Complete sets 1..10^5 for p in {7, 13, 19, 31}: the oracle's batch equals enumerate_cpu."""
    for case in golden('small_sets.json'):
        g = oracle.Geometry(case['p'], case['lo'], case['hi'], case['A'], case['B'])
        assert g.residuals == case['residual_order']
        fa, fb = oracle.OracleFocus(g, 'A'), oracle.OracleFocus(g, 'B')
        width = -(-g.B // 64)
        r = oracle.batch(g, fa, fb, 0, g.B, width=width, output_cap=1 << 20)
        values = sorted(int(n) for n in r['all_values'])
        assert len(values) == case['count']
        assert oracle.digest([str(n) for n in values]) == case['values_sha256']
        assert [n for n in values if oracle.is_cube(n)] == case['cubes']


def test_p67_prefix_matches_enumerate_cpu(oracle):
    case = golden('p67_prefix.json')
    g = oracle.Geometry(67, 1, 10**13, case['A'], case['B'])
    fa, fb = oracle.OracleFocus(g, 'A'), oracle.OracleFocus(g, 'B')
    r = oracle.batch(g, fa, fb, 0, case['v_end'], width=case['v_end'], output_cap=1 << 21)
    values = sorted(int(n) for n in r['all_values'])
    assert len(values) == case['count']
    assert oracle.digest([str(n) for n in values]) == case['values_sha256']


def test_wide_limbs_match_reference(oracle):
    fx = golden('wide.json')
    rand = random.Random(fx['seed'])
    cases = [tuple(int(x) for x in c) for c in fx['edge']]
    cases += [tuple(rand.getrandbits(64) for _ in range(4)) for _ in range(fx['random'])]
    out = oracle.wide(np.array(cases, dtype=np.uint64))
    h = hashlib.sha256()
    for row in out:
        h.update(f'{int(row[0])},{int(row[1])},{int(row[2])};'.encode())
    assert h.hexdigest() == fx['sha256']


def test_plain_and_masked_oracle_agree(oracle, oracle619):
    """The oracle's plain per-position matcher and its masked matcher give the same populations."""
    g, fa, fb = oracle619
    first, end = 100_000_000, 200_000_000
    lo_u, hi_u = g.u_interval(first)[0], g.u_interval(end - 1)[1]
    us, vs = fa.window(lo_u, hi_u), fb.window(first, end)
    plain = oracle.plain_tile(g, us, vs)
    masked = oracle.batch(g, fa, fb, first, end, width=end - first)
    ng = len(g.filter_groups)
    assert plain['populations'][0] == masked['valid_focused_candidates']
    assert plain['populations'][1:ng + 1] == masked['group_survivors']
    assert [str(n) for n in plain['values']] == masked['all_values']


@pytest.mark.parametrize('low,high', [(0, 0), (5, 5), (0, 1), (3, 200)])
def test_small_window_edges(oracle, low, high):
    g = oracle.Geometry(31, 0, 100000, 14 * 19, 9 * 13 * 31)
    f = oracle.OracleFocus(g, 'A')
    got = f.window(low, high).tolist()
    rings = g.rings('A')
    want = [y for y in range(low, high) if all(y % q in r for q, r in rings)]
    assert got == want


def test_p67_whole_domain_figures(oracle):
    """The oracle over 1 < x <= 10^13 at p=67 with A = 2523326, B = 2486169 (v in [0, B) in 64
    slices): positions, group populations, survivor count and digests (ascending numeric order,
    and ascending string order as an independent probe recorded it)."""
    A, B = 2523326, 2486169
    g = oracle.Geometry(67, 1, 10**13, A, B)
    fa, fb = oracle.OracleFocus(g, 'A'), oracle.OracleFocus(g, 'B')
    primes_arr, table = g.residual_arrays()
    ng = len(g.filter_groups)
    chunks, positions, groups = [], 0, np.zeros(ng, dtype=np.uint64)
    step = -(-B // 64)
    for first in range(0, B, step):
        end = min(first + step, B)
        (_, _, ulo, uhi), = g.tile_ranges(first, end, end - first)
        us, vs = fa.window(ulo, uhi, cap=1 << 40), fb.window(first, end, cap=1 << 40)
        counts = np.zeros(ng + 3, dtype=np.uint64)
        cap = 4_000_000
        out = np.zeros(2 * cap, dtype=np.uint64)
        assert oracle.lib().oc_masked_batch(us, len(us), vs, len(vs), A, B, 1, 0, 10**13, 0, primes_arr,
                                            len(g.residuals), table, first, end - first, 1, cap, counts, out,
                                            os.cpu_count() or 1) == 0
        n = int(counts[ng + 1])
        assert n <= cap and not counts[ng + 2]
        chunks.append(out[:2 * n].reshape(-1, 2)[:, 0].copy())
        positions += int(counts[0])
        groups += counts[1:ng + 1]
    values = np.sort(np.concatenate(chunks))
    assert positions == 113_117_444 and groups.tolist() == [74_055_342, 66_984_666, 65_848_989]
    assert len(values) == 65_848_989
    assert oracle.strings_digest_u64(values) == '55ba793e8e7ad01a69ec2948d21f8ed5167ac7042b6c21394e8519c7924a69f9'
    full = ('[' + ','.join('"%s"' % s for s in sorted(map(str, values.tolist()))) + ']\n').encode()
    assert hashlib.sha256(full).hexdigest() == 'f3f1296a795a66e550f16c516d8c752411db58e1b94506b9ff039551ad346587'
