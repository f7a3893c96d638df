"""Host-side logic of the product package against the reference's fixtures (no GPU)."""
from __future__ import annotations

import ctypes
import hashlib
import json
import re

import numpy as np
import pytest

from conftest import ROOT, golden
from psuedocubes_b200 import _native as N
from psuedocubes_b200.accounting import digest, encoded
from psuedocubes_b200.batch_experiment import split_outputs, tile_ranges
from psuedocubes_b200.focus import A619, B619, Config, Tile, targeted_coordinates
from psuedocubes_b200.gpu import launch_plan
from psuedocubes_b200.multi import validate_result
from psuedocubes_b200.optimized import BATCH_WIDTH, Accumulator
from psuedocubes_b200.predicate import icbrt, is_perfect_cube, local3, qualifies3
from psuedocubes_b200.tables import allowed, definition, packed, sieve_primes
from psuedocubes_b200.verify import verify


def test_library_exports_every_declared_symbol():
    header = (ROOT / 'include' / 'pcube.h').read_text()
    declared = set(re.findall(r'^\s*(?:int|const char \*)\s*(pc_\w+)\s*\(', header, re.M))
    assert declared == set(N.SYMBOLS)
    lib = N.lib()
    for name in declared:
        assert hasattr(lib, name), name
    assert lib.pc_version() == 1


def test_tables_and_predicate():
    t = golden('tables.json')
    assert definition(619)['sha256'] == t['sha256_619']
    assert definition(67)['sha256'] == t['sha256_67']
    assert list(allowed(31)) == t['allowed_31'] and list(allowed(9)) == t['allowed_9']
    cubic = [q for q in sieve_primes(619) if q % 3 == 1]
    assert (len(sieve_primes(619)), len(cubic), sum(cubic)) == (114, 54, 15744)
    assert sum(4 * len(packed(q)) for q in cubic) == t['packed_cubic_bytes_619'] == 2076
    known = golden('known.json')
    assert icbrt(3 * 10**27) == known['icbrt_3e27']
    assert local3(int(known['cases'][0]['n']), 619) == known['n613_local3_619']
    for case in known['cases']:
        n, p = int(case['n']), case['p']
        assert local3(n, p) == case['local3'] and is_perfect_cube(n) == case['cube']
        assert verify(n, p) == case['verify']
    for bad in (2, 3, 5, 9, 15, 25, -7):
        with pytest.raises(ValueError):
            local3(1, bad)
    assert local3(1, 619) and not qualifies3(1, 619)


def test_geometry_matches_reference(p619):
    g = golden('geometry.json')
    assert p619.manifest() == g['manifest_619']
    assert p619.filter_order() == g['residual_order_619']
    af, bf = p619.focuses()
    assert [[q, list(r)] for q, r in af.rings] == g['focus_rings_619']['A']
    assert [[q, list(r)] for q, r in bf.rings] == g['focus_rings_619']['B']
    for n, u, v, lo, hi in g['canonical']:
        assert p619.canonical(int(n)) == (int(u), int(v))
        assert p619.u_interval(int(v)) == (int(lo), int(hi))
    for case in g['tile_ranges']:
        rows = tile_ranges(p619, int(case['first']), int(case['end']), case['width'])
        assert [[str(x) for x in row] for row in rows] == case['rows']
    with pytest.raises(ValueError):
        tile_ranges(p619, 0, 65, 1)
    with pytest.raises(ValueError):
        tile_ranges(p619, 0, 1, 0)


def test_small_manifests_match_reference():
    for case in golden('small_sets.json'):
        c = Config(case['p'], case['lo'], case['hi'], case['A'], case['B'])
        assert c.manifest() == case['manifest']
        assert c.filter_order() == case['residual_order']
    case = golden('p67_prefix.json')
    assert Config(67, 1, 10**13, case['A'], case['B']).manifest() == case['manifest']


def test_targeted_coordinates_match_reference():
    for case in golden('known.json')['cases']:
        n, p = int(case['n']), case['p']
        c = Config(p, max(0, n - 100), min(3 * 10**27, n + 100), A619, B619)
        us, vs = targeted_coordinates(c, n)
        assert [str(x) for x in us] == case['us'] and [str(x) for x in vs] == case['vs']
        assert [str(x) for x in c.canonical(n)] == case['canonical']


def test_config_rejections():
    with pytest.raises(ValueError):
        Config(7, 0, 100000, 14, 9 * 13)
    with pytest.raises(ValueError):
        Config(7, 0, 100000, 3 * 7, 3)
    with pytest.raises(ValueError):
        Tile(5, 5).validate(Config(619, 10**27, 3 * 10**27, A619, B619))


def test_encoded_is_canonical():
    assert encoded({'b': 1, 'a': [1 << 53, 2]}) == b'{"a":["9007199254740992",2],"b":1}\n'
    assert digest([]) == '37517e5f3dc66819f61f5a7bb8ace1921282415f10551d2defa5c3eb0985b570'


def test_launch_plan_partitions_every_candidate():
    for nu in (0, 1, 31, 32, 33, 63, 255, 256, 257, 6001):
        for nv in (0, 1, 7, 8, 9, 86, 289, 962):
            for target in (1, 2, 4):
                blocks, stripes = launch_plan(nu, nv, 84, 'warp', target)
                assert bool(blocks) == bool(nu and nv)
                if blocks:
                    assert blocks * 8 >= nv * stripes and blocks * 8 - nv * stripes < 8
    assert launch_plan(6001, 86, 84, 'serial') == (1, 1)
    for layout, target in (('unknown', 2), ('warp', 0), ('warp', True), ('warp', 3)):
        with pytest.raises(ValueError):
            launch_plan(10, 10, 84, layout, target)


def test_split_outputs_groups_and_sorts():
    x1, x2, x3 = 10**27 + 7, 10**27 + 3, 2 * 10**27 + 11
    recs = np.array([[x & (2**64 - 1), (x >> 64) | (t << 32)] for x, t in ((x1, 1), (x2, 1), (x3, 0))],
                    dtype=np.uint64)
    assert split_outputs(recs, 3) == [[x3], [x2, x1], []]


def test_accumulator_rejects_gaps_and_bad_receipts():
    acc = Accumulator(0, 2 * BATCH_WIDTH)
    with pytest.raises(ValueError):
        acc.add(BATCH_WIDTH, 2 * BATCH_WIDTH, {})
    with pytest.raises(ValueError):
        validate_result(0, 10, dict(status='FAIL'))
    with pytest.raises(ValueError):
        validate_result(0, 10, dict(status='PASS', host_verified=True,
                                    subtile_scopes=[dict(first='0', end='5')], valid_focused_candidates=0,
                                    genuine_cubes=0))
    with pytest.raises(ValueError):
        Accumulator(0, 0)


def test_status_codes_map_to_reference_exceptions():
    for code, exc in ((N.PC_OVERFLOW, OverflowError), (N.PC_INVALID, ValueError), (N.PC_ARITHMETIC, ArithmeticError),
                      (N.PC_TIMEOUT, TimeoutError), (N.PC_NOMEM, MemoryError), (N.PC_CUDA, RuntimeError)):
        with pytest.raises(exc):
            N.raise_for(code, None, 'x')
    N.raise_for(N.PC_OK)


def test_scope_encoding_matches_canonical_json():
    """The transcript bytes built from counter arrays equal encoded() of the scope dicts, including
    counters at and above 2^53 (which the canonical form writes as strings)."""
    import random
    from psuedocubes_b200.accounting import EMPTY_DIGEST, digest, encoded, encoded_scopes, scope_list
    assert EMPTY_DIGEST == digest([]) == '37517e5f3dc66819f61f5a7bb8ace1921282415f10551d2defa5c3eb0985b570'
    rng = random.Random(619)
    for trial in range(60):
        n, ng = rng.randint(0, 70), rng.randint(0, 24)
        top = (1 << 53) + 5 if trial % 4 == 0 else 10**9
        firsts = sorted(rng.randrange(0, 10**18) for _ in range(n))
        ends = [f + rng.randrange(1, 10**8) for f in firsts]
        valid = [rng.randrange(0, top) for _ in range(n)]
        groups = [[rng.randrange(0, top) for _ in range(ng)] for _ in range(n)]
        local = [rng.randrange(0, 9000) for _ in range(n)]
        digests = [rng.choice([EMPTY_DIGEST, digest([str(rng.randrange(10**27))])]) for _ in range(n)]
        safe = top < 1 << 53
        scopes = scope_list(firsts, ends, valid, groups, local, digests, below_2_53=safe and trial % 2 == 1)
        assert encoded_scopes(scopes) == encoded(list(scopes))
        assert list(scopes) == [dict(first=str(f), end=str(e), valid_focused_candidates=v, group_survivors=g,
                                     local_survivors=k, output_sha256=d)
                                for f, e, v, g, k, d in zip(firsts, ends, valid, groups, local, digests)]


def test_library_scope_json_equals_canonical_encoding():
    """pc_scopes_json (host-only, no device) writes, batch after batch, exactly the bytes of
    encoded(subtile_scopes) that the lease transcript hashes, including a partial last batch and
    subtile and counters of 2^53 and above."""
    import ctypes
    import random
    from psuedocubes_b200 import _native as N
    from psuedocubes_b200.accounting import EMPTY_DIGEST, digest, encoded
    lib = N.lib()
    rng = random.Random(61)
    for first, batches, tail, ng in ((575222931200000000, 3, 12345, 24), (0, 1, 0, 3), (10**17, 2, 6_400_000_000 - 1, 1)):
        width, per = 100_000_000, 64
        end = first + batches * width * per + tail
        nt = (end - first + width - 1) // width
        counts = np.zeros((nt, ng + 3), dtype=np.uint64)
        top = (1 << 53) + 9
        for t in range(nt):
            counts[t, 0] = rng.randrange(0, top)
            counts[t, 1:ng + 1] = [rng.randrange(0, top if t % 5 == 0 else 10**6) for _ in range(ng)]
            counts[t, ng + 1] = rng.randrange(0, 3)
        digests = [EMPTY_DIGEST if counts[t, ng + 1] == 0 else digest([str(t)]) for t in range(nt)]
        want = b''
        for b0 in range(first, end, width * per):
            b1 = min(b0 + width * per, end)
            scopes = []
            for v in range(b0, b1, width):
                t = (v - first) // width
                scopes.append(dict(first=str(v), end=str(min(v + width, b1)), valid_focused_candidates=int(counts[t, 0]),
                                   group_survivors=[int(x) for x in counts[t, 1:ng + 1]],
                                   local_survivors=int(counts[t, ng + 1]), output_sha256=digests[t]))
            want += encoded(scopes)
        cap = len(want) + 16
        buf = ctypes.create_string_buffer(cap)
        size = ctypes.c_uint64()
        assert lib.pc_scopes_json(counts.reshape(-1), ng + 3, ng, nt, first, end, width, per, ''.join(digests).encode(),
                                  ctypes.addressof(buf), cap, ctypes.byref(size)) == 0
        assert buf.raw[:size.value] == want
        assert lib.pc_scopes_json(counts.reshape(-1), ng + 3, ng, nt, first, end, width, per, ''.join(digests).encode(),
                                  ctypes.addressof(buf), len(want) - 1, ctypes.byref(size)) == N.PC_OVERFLOW
        assert lib.pc_scopes_json(counts.reshape(-1), ng + 3, ng, nt + 1, first, end, width, per,
                                  ''.join(digests).encode(), ctypes.addressof(buf), cap, ctypes.byref(size)) == N.PC_INVALID


def test_overlapped_leases_issue_ahead_and_keep_order(p619):
    """compute_leases issues lease k + 1 to the device before it returns the receipt of lease k,
    keeps one device call in flight, yields receipts in lease order equal to compute_lease's, and
    passes a device error through to the caller."""
    import threading
    import time
    import types
    from psuedocubes_b200.optimized import PROFILE, compute_lease, compute_leases
    width, fg = PROFILE['tile_width'], p619.filter_groups()
    ng = len(fg)
    events, lock, busy = [], threading.Lock(), [0]

    class FakeLeases:
        config, filter_groups = p619, fg
        runtime = types.SimpleNamespace(lib=N.lib())

        def run_lease(self, af, bf, first, end, w):
            with lock:
                busy[0] += 1
                assert busy[0] == 1
                events.append(('run', first))
            if first == 666:
                busy[0] -= 1
                raise ArithmeticError('device failure')
            nt = (end - first + w - 1) // w
            counts = np.zeros((nt, ng + 3), dtype=np.uint64)
            counts[:, 0] = np.arange(nt, dtype=np.uint64) + first % 1000
            counts[:, 1] = counts[:, 0] // 2
            geometry = np.ones((nt, 2), dtype=np.uint64)
            with lock:
                busy[0] -= 1
            return dict(counts=counts, geometry=geometry, per_tile=[[] for _ in range(nt)],
                        stats=dict(kernel_ms=1.0, window_ms=0.5, bounds_ms=0.25))

    leases = [(0, BATCH_WIDTH + 5), (10**17, 10**17 + 3 * width), (5 * BATCH_WIDTH, 6 * BATCH_WIDTH)]
    got = []
    for k, receipt in enumerate(compute_leases(FakeLeases(), None, None, leases)):
        # the generator is suspended here, so the next lease can only run if it was issued already
        if k + 1 < len(leases):
            deadline = time.monotonic() + 10
            while ('run', leases[k + 1][0]) not in events and time.monotonic() < deadline:
                time.sleep(0.001)
            assert ('run', leases[k + 1][0]) in events
        events.append(('receipt', int(receipt['subtile_scopes'][0]['first'])))
        got.append(receipt)
    assert [e for e in events if e[0] == 'receipt'] == [('receipt', f) for f, _ in leases]
    assert [e for e in events if e[0] == 'run'] == [('run', f) for f, _ in leases]
    strip = lambda r: {k: v for k, v in r.items() if not k.endswith('_seconds')}
    for (first, end), receipt in zip(leases, got):
        assert strip(receipt) == strip(compute_lease(FakeLeases(), None, None, first, end))
    with pytest.raises(ArithmeticError):
        list(compute_leases(FakeLeases(), None, None, [(0, width), (666, 666 + width)]))


def test_focus_module_matches_reference_fixtures():
    """Config, Focus, Tile and factors against the reference's pseudocube.focus on five
    configurations (tests/golden/focus.json, written by make_golden.py from the reference)."""
    from psuedocubes_b200.focus import Tile, factors
    fx = golden('focus.json')
    for row in fx['configs']:
        c = Config(row['p'], int(row['lo']), int(row['hi']), int(row['A']), int(row['B']))
        assert c.manifest() == row['manifest'] and c.residuals() == row['residuals']
        for focus, want in zip(c.focuses(), row['foci']):
            assert str(focus.modulus) == want['modulus'] and str(focus.count) == want['count']
            assert [[q, list(r)] for q, r in focus.rings] == want['rings']
            terms = hashlib.sha256(json.dumps([[str(t) for t in ts] for ts in focus.terms]).encode()).hexdigest()
            assert terms == want['terms_sha256']
            first, second = focus.halves()
            assert [[len(t) for t in first], [len(t) for t in second]] == want['halves']
            for i, v in want['at']:
                assert str(focus.at(int(i))) == v
            for x, (period, index) in want['rank']:
                assert focus.rank(int(x)) == (int(period), int(index))
                assert focus.contains(int(x))
            w = want['indices']
            assert [str(x) for x in focus.indices(w['start'], w['end'], w['period'])] == w['values']
        for n, u, v, lo, hi in row['canonical']:
            assert c.canonical(int(n)) == (int(u), int(v)) and c.u_interval(int(v)) == (int(lo), int(hi))
        t = Tile(int(row['tile']['first']), int(row['tile']['end']))
        assert t.manifest(c) == row['tile']['manifest']
        assert [[str(x.first), str(x.end)] for x in t.split()] == row['tile']['split']
    for case in fx['factors']:
        if 'rings' in case:
            assert factors(int(case['n']), case['p']) == case['rings']
        else:
            with pytest.raises(ValueError, match=re.escape(case['error'])):
                factors(int(case['n']), case['p'])
