"""Shared test setup: the `gpu` marker, repository paths, and the device fixtures."""
from __future__ import annotations

import json
import os
import sys
import time
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / 'tests' / 'golden'
#: the reference project's tree; the CPU tests that import its unchanged host code skip without it
REFERENCE = Path(os.environ.get('PSUEDOCUBES_REFERENCE', '/root/reference'))
sys.path.insert(0, str(ROOT))


def pytest_configure(config: pytest.Config) -> None:
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200, sm_100a)')
    config.addinivalue_line('markers', 'slow: long-running CPU check')


def golden(name: str):
    return json.loads((GOLDEN / name).read_text())


@pytest.fixture(scope='session')
def oracle():
    from oracle import pcube_oracle as O
    O.lib()
    return O


@pytest.fixture(scope='session')
def runtime():
    from psuedocubes_b200 import _native as N
    N.lib()  # the extension must exist; a missing library is a failure, not a skip
    if N.device_count() < 1:
        pytest.skip('no CUDA device visible')
    from psuedocubes_b200.gpu import Runtime
    rt = Runtime(time.monotonic() + 3600, 8 * 1024**3)
    yield rt
    rt.close()


@pytest.fixture(scope='session')
def p619():
    from psuedocubes_b200.focus import A619, B619, Config
    return Config(619, 10**27, 3 * 10**27, A619, B619)


@pytest.fixture(scope='session')
def focuses619(runtime, p619):
    from psuedocubes_b200.gpu import GPUFocus
    af, bf = p619.focuses()
    return GPUFocus(runtime, af), GPUFocus(runtime, bf)


@pytest.fixture(scope='session')
def oracle619(oracle):
    g = oracle.Geometry(619, 10**27, 3 * 10**27, oracle.A619, oracle.B619)
    return g, oracle.OracleFocus(g, 'A'), oracle.OracleFocus(g, 'B')
