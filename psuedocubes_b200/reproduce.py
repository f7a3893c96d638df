"""Bounded, portable GPU reproduction; produces no production coverage.

Mirrors tools/reproduce.py:20-61: ``python -m psuedocubes_b200.reproduce --first F --batches N
[--compare-baseline] --output PATH``.  Same bounds (1 <= N <= 256, 0 <= F < B), one visible GPU,
180 s deadline, 8 GiB device cap, refuses an existing output, compares the lease against the plain
per-tile matcher by digest of every non-timing field, writes the record durably and prints one
JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import time
from pathlib import Path

from .accounting import digest, durable
from .batch_experiment import MaskedMatcher
from .focus import A619, B619, Config
from .gpu import GPUFocus, Matcher, Runtime, device_count
from .optimized import Accumulator, BATCH_WIDTH, compute_lease
from .run_production import compute_batch


def main(argv: list[str] | None = None) -> dict:
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument('--first', type=int, default=0)
    parser.add_argument('--batches', type=int, default=1)
    parser.add_argument('--compare-baseline', action='store_true')
    parser.add_argument('--output', type=Path, required=True)
    args = parser.parse_args(argv)
    if not 1 <= args.batches <= 256 or not 0 <= args.first < B619:
        raise ValueError('bounded canonical scope required')
    if args.output.exists():
        raise ValueError('choose a new output path to retain previous evidence')
    visible = os.environ.get('CUDA_VISIBLE_DEVICES')
    if not visible or ',' in visible:
        raise ValueError('select one available GPU with CUDA_VISIBLE_DEVICES')
    config = Config(619, 10**27, 3 * 10**27, A619, B619)
    end = min(B619, args.first + args.batches * BATCH_WIDTH)
    runtime = Runtime(time.monotonic() + 180, 8 * 1024**3)
    if device_count() != 1:
        raise ValueError('exactly one visible device required')
    af, bf = (GPUFocus(runtime, f) for f in config.focuses())
    result = compute_lease(MaskedMatcher(runtime, config), af, bf, args.first, end)
    baseline_seconds = None
    if args.compare_baseline:
        reference = Matcher(runtime, config)
        accumulator = Accumulator(args.first, end)
        started = time.monotonic()
        for first in range(args.first, end, BATCH_WIDTH):
            stop = min(first + BATCH_WIDTH, end)
            accumulator.add(first, stop, compute_batch(reference, af, bf, first, stop, 100_000_000))
        baseline = accumulator.finish(time.monotonic() - started)
        expected = {k: v for k, v in baseline.items() if not k.endswith('_seconds')}
        actual = {k: v for k, v in result.items() if not k.endswith('_seconds')}
        if digest(expected) != digest(actual):
            raise ArithmeticError('complete batch/reference mismatch')
        baseline_seconds = baseline['elapsed_seconds']
    record = dict(status='PASS', production_coverage=0, first=str(args.first), end=str(end),
                  baseline_compared=args.compare_baseline, baseline_seconds=baseline_seconds, result=result,
                  source_manifest=dict(library=runtime.compiles[0]['source_sha256']),
                  peak_device_bytes=runtime.peak_device, compiled_kernels=runtime.compiles)
    durable(args.output, record)
    line = dict(status='PASS', output=str(args.output), production_coverage=0,
                candidates=result['valid_focused_candidates'], seconds=result['elapsed_seconds'],
                baseline_seconds=baseline_seconds)
    print(json.dumps(line))
    return record


if __name__ == '__main__':
    main()
