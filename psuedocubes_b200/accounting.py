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
    return hashlib.sha256(encoded(value)).hexdigest()


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
