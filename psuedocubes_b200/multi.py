"""Receipt validation of the shared frontier (mirrors pseudocube/multi.py:36-71).

Only ``validate_result`` and ``subtile_count`` live here: the SQLite frontier that consumes
receipts stays a host-side component outside the GPU path.
"""
from __future__ import annotations

from typing import Any

from .accounting import digest

HEX = set('0123456789abcdef')


def validate_result(first: int, end: int, result: dict[str, Any]) -> None:
    """Reject any receipt that cannot become coverage of [first, end)."""
    if (result.get('status') != 'PASS' or result.get('host_verified') is not True
            or result.get('overflow') or result.get('kernel_error')):
        raise ValueError('unverified execution cannot become coverage')
    cursor = first
    for tile in result['subtile_scopes']:
        if int(tile['first']) != cursor or not cursor < int(tile['end']) <= end:
            raise ValueError('gap or overlap in execution subtiles')
        cursor = int(tile['end'])
    if cursor != end:
        raise ValueError('incomplete execution receipt')
    for key in ('valid_focused_candidates', 'genuine_cubes'):
        if int(result[key]) < 0:
            raise ValueError('negative execution count')
    fmt = result.get('receipt_format')
    if fmt == 'compact-batch-v1':
        width = int(result['tile_width'])
        batch = int(result['compute_batch_width'])
        if width <= 0 or batch != 64 * width or len(result['subtile_scopes']) != 1:
            raise ValueError('invalid compact execution geometry')
        if int(result['subtiles_executed']) != (end - first + width - 1) // width:
            raise ValueError('compact subtile count mismatch')
        if int(result['compute_batches']) != (end - first + batch - 1) // batch:
            raise ValueError('compact batch count mismatch')
        transcript = result['subtile_scopes'][0]['transcript_sha256']
        if len(transcript) != 64 or any(ch not in HEX for ch in transcript):
            raise ValueError('invalid execution transcript hash')
        values = result['all_values']
        if len(values) != len(set(values)) or len(values) != int(result['genuine_cubes']) + len(result['cpu_confirmed_hits']):
            raise ValueError('compact output count mismatch')
        if result['subtile_scopes'][0]['output_sha256'] != digest(values):
            raise ValueError('compact output hash mismatch')
    elif 'subtiles_executed' in result or fmt is not None:
        raise ValueError('unknown receipt format')


def subtile_count(result: dict[str, Any]) -> int:
    return int(result.get('subtiles_executed', len(result['subtile_scopes'])))
