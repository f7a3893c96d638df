"""Plain per-tile batch over the plain matcher (mirrors tools/run_production.py:51-83).

The per-10^8 tile loop the reference's ``--compare-baseline`` and plain production service use:
each tile runs the plain matcher; an OverflowError splits the tile and replays both halves.
"""
from __future__ import annotations

import time
from typing import Any

from .accounting import digest
from .focus import Tile
from .gpu import GPUFocus, Matcher
from .verify import verify


def compute_batch(matcher: Matcher, af: GPUFocus, bf: GPUFocus, first: int, end: int, width: int) -> dict[str, Any]:
    started = time.monotonic()
    scopes: list[dict[str, Any]] = []
    hits: list[dict[str, Any]] = []
    values: list[str] = []
    groups = [0] * len(matcher.filter_groups)
    counts = dict.fromkeys(('focus_u', 'focus_v', 'cartesian_opportunities', 'valid_focused_candidates',
                            'genuine_cubes', 'local_survivors', 'cube_checks'), 0)
    timings = dict.fromkeys(('kernel_seconds', 'focus_enumeration_seconds', 'transfer_seconds',
                             'verification_seconds'), 0.0)
    overflow_splits: list[dict[str, str]] = []

    def execute(tile: Tile) -> None:
        try:
            row = matcher.tile(tile, af, bf)
        except OverflowError:
            if tile.end - tile.first < 2:
                raise
            overflow_splits.append(dict(first=str(tile.first), end=str(tile.end)))
            left, right = tile.split()
            execute(left)
            execute(right)
            return
        if row['status'] != 'PASS' or not row['host_verified'] or row['cpu_rejected_reports']:
            raise ArithmeticError('unverified GPU tile')
        for n in row['cpu_confirmed_hits']:
            witness = verify(int(n), matcher.config.p)
            if not witness['valid_pseudocube']:
                raise ArithmeticError('standalone candidate verification failed')
            hits.append(witness)
        scopes.append(dict(first=str(tile.first), end=str(tile.end),
                           valid_focused_candidates=row['valid_focused_candidates'],
                           group_survivors=row['group_survivors'], local_survivors=row['local_survivors'],
                           output_sha256=digest(row['all_values'])))
        values.extend(row['all_values'])
        for key in counts:
            counts[key] += int(row[key])
        for key in timings:
            timings[key] += float(row[key])
        for i, value in enumerate(row['group_survivors']):
            groups[i] += value

    for start in range(first, end, width):
        execute(Tile(start, min(start + width, end)))
    if len(values) != len(set(values)):
        raise ArithmeticError('duplicate output across disjoint subtiles')
    return dict(status='PASS', host_verified=True, **counts, **timings, subtile_scopes=scopes,
                filter_groups=matcher.filter_groups, group_survivors=groups, all_values=values,
                cpu_confirmed_hits=hits, overflow_splits=overflow_splits,
                elapsed_seconds=time.monotonic() - started,
                claim='Executed primary coverage; independent replay required before any minimum claim.')
