"""Regenerate the golden fixtures in this directory from the reference project.

Run from the repository root with the path of the reference project's tree:

    python tests/golden/make_golden.py <reference tree>
    python tests/golden/make_golden.py <reference tree> --cube-roots-only    # cube_roots.json alone
    python tests/golden/make_golden.py <reference tree> --focus-only         # focus.json alone

It imports the reference's own Python (pseudocube.focus / oracle / tables / accounting,
review.verify_cube) from a scratch copy, runs the reference's compiled review tools from
oracle/_ref (focus_window_cpu.cpp, wide.c; built by oracle/Makefile), and reads the reference's
golden lease replay.  The fixtures are small JSON files; nothing here runs at test time.
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import random
import shutil
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]


def dump(name: str, value: object) -> None:
    (HERE / name).write_text(json.dumps(value, indent=1, sort_keys=True) + '\n')
    print('wrote', name)


def cube_root_fixtures(reference: Path) -> None:
    """Genuine-cube control: the reference's recorded full-interval count
    (results/completion-2026-09-16/cube_count*.json) and its two compiled checkers
    (review/cube_count.c, review/cube_count_independent.c, built into oracle/_ref) on list and
    count cases; the two checkers must agree on every case."""
    import subprocess

    def run(name: str, a: int, b: int, p: int, listed: bool) -> dict:
        cmd = [str(ROOT / 'oracle/_ref' / name), str(a), str(b), str(p)] + (['--list'] if listed else [])
        return json.loads(subprocess.check_output(cmd, text=True))

    recorded = []
    for name in ('cube_count', 'cube_count_independent'):
        row = json.loads((reference / f'results/completion-2026-09-16/{name}.json').read_text())
        recorded.append(dict(checker=name, algorithm=row['algorithm'], first=int(row['root_first']),
                             last=int(row['root_last']), p=int(row['p']), count=int(row['count']),
                             source=f'results/completion-2026-09-16/{name}.json'))
    listed = []
    for a, b, p in ((1, 1000, 7), (1, 1000, 2), (1, 1000, 3), (2, 2, 2), (1, 1, 2000), (1, 100000, 619),
                    (1000000001, 1000100000, 619), (1442149571, 1442249570, 619), (4294867296, 4294967295, 619),
                    (999999937, 1000099936, 1999), (3, 34, 31)):
        rows = [run(name, a, b, p, True) for name in ('cube_count', 'cube_count_independent')]
        assert rows[0]['roots'] == rows[1]['roots'] and rows[0]['count'] == rows[1]['count']
        roots = rows[0]['roots']
        listed.append(dict(first=a, last=b, p=p, count=int(rows[0]['count']), head=[int(x) for x in roots[:16]],
                           tail=[int(x) for x in roots[-16:]],
                           sha256=hashlib.sha256(','.join(roots).encode()).hexdigest()))
    counted = []
    for a, b, p in ((1, 10**7, 619), (123456789, 133456789, 1999), (4000000000, 4294967295, 619),
                    (1, 4294967295, 2), (1000000001, 1442249570, 5), (1000000001, 1442249570, 97),
                    (1000000001, 1442249570, 2000), (7, 7, 5), (1, 2**20 + 17, 619)):
        rows = [run(name, a, b, p, False) for name in ('cube_count', 'cube_count_independent')]
        assert rows[0]['count'] == rows[1]['count']
        counted.append(dict(first=a, last=b, p=p, count=int(rows[0]['count'])))
    dump('cube_roots.json', dict(recorded=recorded, listed=listed, counted=counted,
                                 list_digest='sha256 of the ascending decimal roots joined by commas'))


def focus_fixtures(reference: Path) -> None:
    """The reference's pseudocube.focus on five configurations (p = 619 production, the p = 67
    split, the p = 31, 13 and 7 small sets): manifests, filter order, rings, terms digests, halves,
    seeded at/rank/indices samples, canonical pairs, u intervals, tile manifests and splits, and
    factors() answers (ring moduli or the error message) on accepted and refused moduli."""
    scratch = Path(tempfile.mkdtemp(prefix='pcube-ref-'))
    shutil.copytree(reference / 'pseudocube', scratch / 'pseudocube')
    sys.path.insert(0, str(scratch))
    from pseudocube.focus import A619, B619, Config, Tile, factors
    rng = random.Random(619003)
    configs = []
    for p, lo, hi, A, B in ((619, 10**27, 3 * 10**27, A619, B619), (67, 1, 10**13, 2523326, 2486169),
                            (31, 0, 100000, 266, 3627), (13, 0, 100000, 14, 117), (7, 0, 100000, 14, 9)):
        c = Config(p, lo, hi, A, B)
        row = dict(p=p, lo=str(lo), hi=str(hi), A=str(A), B=str(B), manifest=c.manifest(),
                   residuals=c.residuals(), foci=[])
        for focus in c.focuses():
            at = [(i, focus.at(i)) for i in sorted(rng.randrange(focus.count) for _ in range(64))]
            coords = [focus.at(rng.randrange(focus.count)) + rng.randrange(3) * focus.modulus for _ in range(64)]
            start = rng.randrange(max(1, focus.count - 40))
            first, second = focus.halves()
            row['foci'].append(dict(
                modulus=str(focus.modulus), count=str(focus.count), rings=[[q, list(r)] for q, r in focus.rings],
                terms_sha256=hashlib.sha256(json.dumps([[str(t) for t in ts] for ts in focus.terms]).encode()).hexdigest(),
                halves=[[len(t) for t in first], [len(t) for t in second]],
                at=[[str(i), str(v)] for i, v in at], rank=[[str(x), [str(k) for k in focus.rank(x)]] for x in coords],
                indices=dict(start=start, end=min(focus.count, start + 40), period=2,
                             values=[str(x) for x in focus.indices(start, min(focus.count, start + 40), 2)])))
        row['canonical'] = []
        for n in [lo + 1, hi, *(rng.randrange(lo + 1, hi + 1) for _ in range(64))]:
            u, v = c.canonical(n)
            row['canonical'].append([str(n), str(u), str(v), *(str(x) for x in c.u_interval(v))])
        t = Tile(rng.randrange(B // 2), B)
        row['tile'] = dict(first=str(t.first), end=str(t.end), manifest=t.manifest(c),
                           split=[[str(x.first), str(x.end)] for x in t.split()])
        configs.append(row)
    answers = []
    for n, p in ((14, 7), (9, 7), (3, 7), (27 * 5, 7), (9 * 49, 7), (9 * 11, 7), (8 * 7, 13), (10**19, 7),
                 (0, 7), (1, 7), (A619, 619), (B619, 619), (A619, 179), (9 * 7 * 13 * 31, 31)):
        try:
            answers.append(dict(n=str(n), p=p, rings=factors(n, p)))
        except ValueError as exc:
            answers.append(dict(n=str(n), p=p, error=str(exc)))
    dump('focus.json', dict(configs=configs, factors=answers))
    shutil.rmtree(scratch)


def main(reference: Path) -> None:
    sys.dont_write_bytecode = True
    scratch = Path(tempfile.mkdtemp(prefix='pcube-ref-'))
    shutil.copytree(reference / 'pseudocube', scratch / 'pseudocube')
    shutil.copytree(reference / 'review', scratch / 'review')
    shutil.copytree(reference / 'kernels', scratch / 'kernels')
    sys.path.insert(0, str(scratch))
    sys.path.insert(0, str(ROOT))
    from pseudocube.accounting import digest, encoded
    from pseudocube.batch_experiment import tile_ranges
    from pseudocube.focus import A619, B619, Config, Tile, enumerate_cpu, targeted_coordinates
    from pseudocube.oracle import icbrt, is_perfect_cube, local3
    from pseudocube.tables import allowed, definition, packed
    from review.verify_cube import verify
    from oracle import pcube_oracle as O

    # 1. golden lease (results/continuation-2026-09-15/positive-lease-replay.json)
    replay = json.loads((reference / 'results/continuation-2026-09-15/positive-lease-replay.json').read_text())
    r = replay['result']
    keep = ('focus_u', 'focus_v', 'cartesian_opportunities', 'valid_focused_candidates', 'genuine_cubes',
            'local_survivors', 'cube_checks', 'group_survivors', 'filter_groups', 'all_values',
            'cpu_confirmed_hits', 'compute_batches', 'subtiles_executed', 'tile_width', 'compute_batch_width',
            'receipt_format')
    dump('golden_lease.json', dict(first=replay['first'], end=replay['end'],
                                   source='results/continuation-2026-09-15/positive-lease-replay.json',
                                   result={k: r[k] for k in keep},
                                   transcript_sha256=r['subtile_scopes'][0]['transcript_sha256'],
                                   output_sha256=r['subtile_scopes'][0]['output_sha256']))

    # 2. complete small sets (tests/test_pseudocube_math.py:19-20,74-88) via enumerate_cpu
    def small_config(p: int, lo: int = 0, hi: int = 100000) -> Config:
        return Config(p, lo, hi, 14 * (19 if p >= 19 else 1), 9 * (13 if p >= 13 else 1) * (31 if p >= 31 else 1))

    small = []
    for p in (7, 13, 19, 31):
        c = small_config(p)
        values = sorted(enumerate_cpu(c, Tile(0, c.B)))
        residuals = c.residuals()
        residuals.sort(key=lambda q: (q != 9 and q % 3 != 1, q))
        small.append(dict(p=p, lo=c.lo, hi=c.hi, A=c.A, B=c.B, count=len(values),
                          values_sha256=digest([str(n) for n in values]), head=values[:20],
                          cubes=[n for n in values if is_perfect_cube(n)],
                          residual_order=residuals, manifest=c.manifest()))
    dump('small_sets.json', small)

    # 3. p=67 split chosen for the small production-shaped case (1 < x <= 10^13), with the
    #    reference's enumerate_cpu on a v prefix as the cross-check of the oracle
    c67 = Config(67, 1, 10**13, 2523326, 2486169)
    prefix = sorted(enumerate_cpu(c67, Tile(0, 2000)))
    g67 = O.Geometry(67, 1, 10**13, 2523326, 2486169)
    fa, fb = O.OracleFocus(g67, 'A'), O.OracleFocus(g67, 'B')
    oracle_prefix = O.batch(g67, fa, fb, 0, 2000, width=2000, output_cap=1 << 20, verify_values=False)
    assert sorted(int(n) for n in oracle_prefix['all_values']) == prefix, 'p=67 oracle/enumerate_cpu mismatch'
    dump('p67_prefix.json', dict(p=67, lo=1, hi=10**13, A=2523326, B=2486169, v_end=2000, count=len(prefix),
                                 values_sha256=digest([str(n) for n in prefix]), manifest=c67.manifest()))

    # 4. focus windows: reference focus_window_cpu.cpp over half sums of the p=619 focuses,
    #    and the reference's own Focus.window for a small focus
    so = ctypes.CDLL(str(ROOT / 'oracle/_ref/focus_window.so'))
    pointer = np.ctypeslib.ndpointer(dtype=np.uint64, flags='C_CONTIGUOUS')
    so.focus_window.argtypes = [pointer, ctypes.c_uint64, pointer, ctypes.c_uint64, ctypes.c_uint64,
                                ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, pointer, ctypes.c_uint64,
                                ctypes.POINTER(ctypes.c_uint64)]
    config = Config(619, 10**27, 3 * 10**27, A619, B619)
    af, bf = config.focuses()
    windows = []
    for name, focus in (('A', af), ('B', bf)):
        first, second = focus.halves()
        C = np.sort(O.partial([list(t) for t in first], focus.modulus))
        D = np.sort(O.partial([list(t) for t in second], focus.modulus))
        M = focus.modulus

        def ref_window(low: int, high: int) -> list[int]:
            out = []
            for period in range(low // M, (high - 1) // M + 1):
                base = period * M
                a, b = max(0, low - base), min(M, high - base)
                buf = np.zeros(4_000_000, dtype=np.uint64)
                count = ctypes.c_uint64()
                rc = so.focus_window(C, len(C), D, len(D), M, a, b, base, buf, len(buf), ctypes.byref(count))
                assert rc == 0, rc
                out.extend(int(x) for x in buf[:count.value])
            return sorted(out)

        if name == 'A':
            lease_first = 575222931200000000
            cases = [(config.u_interval(0)[0], config.u_interval(6400000000 - 1)[1]),
                     (config.u_interval(lease_first)[0], config.u_interval(lease_first + 6400000000 - 1)[1]),
                     (M - 3_000_000_000, M + 3_000_000_000),
                     (config.u_interval(B619 - 6400000000)[0], config.u_interval(B619 - 1)[1])]
        else:
            cases = [(0, 6400000000), (575222931200000000, 575222931200000000 + 6400000000),
                     (B619 - 6400000000, B619), (B619 // 2, B619 // 2 + 100_000_000)]
        for low, high in cases:
            values = ref_window(low, high)
            windows.append(dict(focus=name, low=str(low), high=str(high), count=len(values),
                                sha256=hashlib.sha256(np.array(values, dtype=np.uint64).tobytes()).hexdigest(),
                                head=[str(x) for x in values[:5]], tail=[str(x) for x in values[-5:]]))
    small_c = small_config(31)
    saf, sbf = small_c.focuses()
    for focus, (low, high) in ((saf, (0, 2000)), (saf, (17, 5 * small_c.A + 3)), (sbf, (0, small_c.B)),
                               (sbf, (100, 2 * small_c.B + 7))):
        values = sorted(focus.window(low, high))   # Focus.window yields in CRT index order
        windows.append(dict(focus='small31-' + ('A' if focus is saf else 'B'), low=str(low), high=str(high),
                            count=len(values), values=[str(x) for x in values][:400],
                            sha256=hashlib.sha256(np.array(values, dtype=np.uint64).tobytes()).hexdigest()))
    dump('windows.json', windows)

    # 5. geometry: tile ranges (tests/test_pseudocube_batch_experiment.py:36-48), canonical pairs and
    #    exact u intervals for seeded x (tests/test_pseudocube_math.py:90-101)
    geometry = dict(tile_ranges=[], canonical=[])
    for first, end, width in ((0, 6400000000, 100000000), (B619 - 6400000000, B619, 100000000),
                              (0, 6400000001, 100000001), (575222931200000000, 575222931200000000 + 6400000000, 100000000)):
        rows = tile_ranges(config, first, end, width)
        geometry['tile_ranges'].append(dict(first=str(first), end=str(end), width=width,
                                            rows=[[str(x) for x in row] for row in rows]))
    rng = random.Random(619003)
    for n in [config.lo, config.lo + 1, config.hi, config.hi + 1, *[rng.randrange(config.lo, config.hi + 1) for _ in range(300)]]:
        u, v = config.canonical(n)
        low, high = config.u_interval(v)
        geometry['canonical'].append([str(n), str(u), str(v), str(low), str(high)])
    geometry['manifest_619'] = config.manifest()
    residuals = config.residuals()
    residuals.sort(key=lambda q: (q != 9 and q % 3 != 1, q))
    geometry['residual_order_619'] = residuals
    geometry['focus_rings_619'] = {'A': [[q, list(res)] for q, res in af.rings], 'B': [[q, list(res)] for q, res in bf.rings]}
    dump('geometry.json', geometry)

    # 6. known answers (tests/test_pseudocube_math.py:103-117; tools/run_production.py:102-105)
    N613 = 674441580981249129037406633
    known = []
    for p, n in ((613, N613), (619, 1000000007**3), (619, 1000000009**3)):
        narrow = Config(p, max(0, n - 100), min(3 * 10**27, n + 100), A619, B619)
        us, vs = targeted_coordinates(narrow, n)
        known.append(dict(p=p, n=str(n), local3=local3(n, p), cube=is_perfect_cube(n), canonical=[str(x) for x in narrow.canonical(n)],
                          us=[str(x) for x in us], vs=[str(x) for x in vs], verify=verify(n, p)))
    dump('known.json', dict(cases=known, n613_local3_619=local3(N613, 619), n613_pow_206_619=pow(N613, 206, 619),
                            icbrt_3e27=icbrt(3 * 10**27)))

    # 7. 128-bit limb cases through the reference's compiled wide.c (seed 619003, 2000 + 5 edge)
    wso = ctypes.CDLL(str(ROOT / 'oracle/_ref/wide.so'))
    wso.products.argtypes = [ctypes.c_uint64] * 4 + [ctypes.POINTER(ctypes.c_uint64)] * 2
    wso.products.restype = ctypes.c_int
    rand = random.Random(619003)
    cases = [(0, 0, 0, 0), (2**64 - 1, 2**64 - 1, 0, 0), (0, 0, 2**64 - 1, 2**64 - 1), (2**32, 2**32, 1, 1), (2**64 - 1, 1, 0, 0)]
    cases += [tuple(rand.getrandbits(64) for _ in range(4)) for _ in range(2000)]
    h = hashlib.sha256()
    for a, b, cc, d in cases:
        low, high = ctypes.c_uint64(), ctypes.c_uint64()
        borrow = wso.products(a, b, cc, d, ctypes.byref(low), ctypes.byref(high))
        h.update(f'{low.value},{high.value},{borrow};'.encode())
    dump('wide.json', dict(seed=619003, edge=[[str(x) for x in case] for case in cases[:5]], random=2000,
                           sha256=h.hexdigest()))

    # 8. residue tables (pseudocube/tables.py)
    dump('tables.json', dict(sha256_619=definition(619)['sha256'], sha256_67=definition(67)['sha256'],
                             packed_cubic_bytes_619=sum(4 * len(packed(q)) for q in range(2, 620)
                                                        if q % 3 == 1 and all(q % d for d in range(2, int(q**0.5) + 1))),
                             allowed_31=list(allowed(31)), allowed_9=list(allowed(9))))
    shutil.rmtree(scratch)
    _ = encoded
    cube_root_fixtures(reference)


if __name__ == '__main__':
    args = [a for a in sys.argv[1:] if not a.startswith('--')]
    if not args:
        raise SystemExit('usage: make_golden.py <reference tree> [--cube-roots-only]')
    ref = Path(args[0])
    if '--cube-roots-only' in sys.argv:
        cube_root_fixtures(ref)
    elif '--focus-only' in sys.argv:
        focus_fixtures(ref)
    else:
        main(ref)
        focus_fixtures(ref)
