"""Canonical JSON, hashes and durable writes (mirrors pseudocube/accounting.py:17-49).

Transcripts and output hashes depend on these bytes, so the encoding is exactly: integers of
magnitude >= 2^53 as decimal strings, sorted keys, no spaces, NaN rejected, trailing newline.
"""
from __future__ import annotations

import hashlib
import json
import os
import uuid
from pathlib import Path
from typing import Any


def interoperable(value: Any) -> Any:
    if type(value) is int and abs(value) >= 1 << 53:
        return str(value)
    if isinstance(value, dict):
        return {str(k): interoperable(v) for k, v in value.items()}
    if isinstance(value, (list, tuple)):
        return [interoperable(v) for v in value]
    return value


def encoded(value: Any) -> bytes:
    text = json.dumps(interoperable(value), sort_keys=True, separators=(',', ':'), allow_nan=False)
    return (text + '\n').encode()


def digest(value: Any) -> str:
    if isinstance(value, list) and not value:
        return EMPTY_DIGEST
    return hashlib.sha256(encoded(value)).hexdigest()


EMPTY_DIGEST = hashlib.sha256(encoded([])).hexdigest()
_SAFE = 1 << 53


class ScopeList(list):
    """A list of subtile scopes that may carry its own canonical encoding (``encoded``), built by
    the producer from the counter arrays; it compares, iterates and serialises as a plain list."""
    encoded: bytes | None = None


def scope_list(firsts: list[int], ends: list[int], valid: list[int], groups: list[list[int]], local: list[int],
               digests: list[str], below_2_53: bool = False) -> ScopeList:
    """Subtile scope dicts of one batch (first/end as decimal strings) with their encoded() bytes
    produced by one %-format per scope; the bytes equal encoded(list of the dicts).  below_2_53:
    the caller has checked that every counter is a non-negative integer below 2^53."""
    out = ScopeList(dict(first=str(f), end=str(e), valid_focused_candidates=v, group_survivors=g, local_survivors=n,
                         output_sha256=d) for f, e, v, g, n, d in zip(firsts, ends, valid, groups, local, digests))
    ng = len(groups[0]) if groups else 0
    if below_2_53 or all(-_SAFE < x < _SAFE for x in (*valid, *local, *(y for g in groups for y in g))):
        fmt = ('{"end":"%d","first":"%d","group_survivors":[' + ','.join(['%d'] * ng) +
               '],"local_survivors":%d,"output_sha256":"%s","valid_focused_candidates":%d}')
        body = ','.join([fmt % (e, f, *g, n, d, v) for f, e, v, g, n, d in zip(firsts, ends, valid, groups, local, digests)])
        out.encoded = ('[' + body + ']\n').encode()
    return out


def encoded_scopes(scopes: list[dict[str, Any]]) -> bytes:
    """encoded(scopes), taken from the list itself when its producer attached the bytes."""
    pre = getattr(scopes, 'encoded', None)
    return pre if pre is not None else encoded(scopes)


def durable(path: Path, value: Any) -> str:
    """Write-then-rename with fsync of the file and its directory; returns the sha256."""
    path.parent.mkdir(parents=True, exist_ok=True)
    data = encoded(value)
    temporary = path.with_name(f'{path.name}.{uuid.uuid4().hex}.tmp')
    with temporary.open('xb') as stream:
        stream.write(data)
        stream.flush()
        os.fsync(stream.fileno())
    os.replace(temporary, path)
    fd = os.open(path.parent, os.O_RDONLY)
    try:
        os.fsync(fd)
    finally:
        os.close(fd)
    return hashlib.sha256(data).hexdigest()
