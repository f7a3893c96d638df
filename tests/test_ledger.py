"""Receipts of this library committed through the reference's own, unchanged ledger code.

The reference's deployed worker (tools/run_multi.py:92-104 of its release archive
releases/20260916-exhaust-v1.tar.gz) loops

    job = frontier.next_batch(device); result = compute_lease(...); frontier.complete(device, job, result)

against its SQLite SharedFrontier (pseudocube/multi.py:197-272), and the single-owner production
service commits through Frontier.complete (pseudocube/production.py:71-108).  This library does
not rebuild either: here both are imported unchanged from a scratch copy of the reference tree,
and this library's receipt of the golden lease (tests/golden/golden_lease_receipt.json, written
from the device path by make_receipt.py and checked against it by test_gpu_parity) is committed
through them and audited.  A tampered receipt must be refused.  Skipped where the reference tree
is absent.
"""
from __future__ import annotations

import copy
import importlib
import shutil
import sys

import pytest

from conftest import REFERENCE, golden
from psuedocubes_b200.focus import B619
from psuedocubes_b200.multi import validate_result as mirror_validate
from psuedocubes_b200.optimized import LEASE_WIDTH, PROFILE

pytestmark = pytest.mark.skipif(not (REFERENCE / 'pseudocube' / 'multi.py').is_file(), reason='reference tree absent')


@pytest.fixture(scope='module')
def ledger(tmp_path_factory):
    scratch = tmp_path_factory.mktemp('reference')
    shutil.copytree(REFERENCE / 'pseudocube', scratch / 'pseudocube')
    sys.path.insert(0, str(scratch))
    try:
        yield importlib.import_module('pseudocube.multi'), importlib.import_module('pseudocube.production')
    finally:
        sys.path.remove(str(scratch))
        for name in [m for m in sys.modules if m == 'pseudocube' or m.startswith('pseudocube.')]:
            del sys.modules[name]


@pytest.fixture(scope='module')
def receipt():
    fx = golden('golden_lease_receipt.json')
    gold = golden('golden_lease.json')
    assert (fx['first'], fx['end']) == (gold['first'], gold['end'])
    assert fx['receipt']['subtile_scopes'][0]['transcript_sha256'] == gold['transcript_sha256']
    return int(fx['first']), int(fx['end']), fx['receipt']


def test_receipt_equals_the_reference_replay_receipt(receipt):
    """Apart from timings, the receipt is the reference's own receipt of the same lease
    (results/continuation-2026-09-15/positive-lease-replay.json)."""
    import json
    first, end, r = receipt
    replay = json.loads((REFERENCE / 'results/continuation-2026-09-15/positive-lease-replay.json').read_text())
    assert (int(replay['first']), int(replay['end'])) == (first, end)
    strip = lambda d: {k: v for k, v in d.items() if not k.endswith('_seconds')}
    assert strip(r) == strip(replay['result'])


def test_receipt_commits_through_the_shared_frontier(ledger, receipt, tmp_path):
    multi, _ = ledger
    first, end, r = receipt
    multi.validate_result(first, end, r)
    mirror_validate(first, end, r)
    baseline = dict(cursor=str(first), campaign_state='searching', commits=0, candidates='0', cubes='0', subtiles=0)
    frontier = multi.SharedFrontier(tmp_path / 'coverage', dict(purpose='receipt check'), 'psuedocubes-b200', B619,
                                    LEASE_WIDTH, multi.DEVICES, baseline, PROFILE)
    device = multi.DEVICES[1]
    job = frontier.next_batch(device)
    assert job[2:] == (first, end)
    frontier.complete(device, job, r)
    audit = frontier.audit_shared()
    assert audit['status'] == 'PASS' and audit['committed_v_end'] == str(end) and not audit['unfinished_leases']
    assert audit['totals'] == dict(commits=1, candidates=r['valid_focused_candidates'], cubes=r['genuine_cubes'],
                                   subtiles=16384)
    assert audit['worker_commits'][device] == 1
    # the golden lease holds one noncube witness, so the campaign stops on it
    assert frontier.state()['campaign_state'] == 'candidate-found'
    assert [row[0] for row in frontier.db.execute('SELECT n FROM candidates')] == [h['n'] for h in r['cpu_confirmed_hits']]
    frontier.validate_owner_receipt(device)
    frontier.db.close()


def test_receipt_commits_through_the_production_frontier(ledger, receipt, tmp_path):
    _, production = ledger
    first, end, r = receipt
    frontier = production.Frontier(tmp_path / 'production', dict(purpose='receipt check'), 'psuedocubes-b200', B619,
                                   LEASE_WIDTH)
    # a frontier whose contiguous cursor has reached the golden lease
    frontier.db.execute("INSERT OR REPLACE INTO meta VALUES('cursor', ?)", (str(first),))
    work, token, start, stop = frontier.next_batch()
    assert (start, stop) == (first, end)
    frontier.complete(work, token, first, end, r)
    state = frontier.state()
    assert state['cursor'] == str(end) and state['commits'] == '1' and state['campaign_state'] == 'candidate-found'
    assert state['candidates'] == str(r['valid_focused_candidates']) and state['cubes'] == str(r['genuine_cubes'])
    frontier.validate_last_receipt()
    frontier.db.close()


def test_tampered_receipts_are_refused(ledger, receipt):
    multi, _ = ledger
    first, end, r = receipt
    cases = []
    bad = copy.deepcopy(r)
    bad['all_values'] = bad['all_values'][1:]                       # a value dropped
    cases.append(bad)
    bad = copy.deepcopy(r)
    bad['subtile_scopes'][0]['output_sha256'] = '0' * 64              # output hash changed
    cases.append(bad)
    bad = copy.deepcopy(r)
    bad['subtiles_executed'] -= 1                                     # geometry changed
    cases.append(bad)
    bad = copy.deepcopy(r)
    bad['host_verified'] = False
    cases.append(bad)
    for bad in cases:
        with pytest.raises(ValueError):
            multi.validate_result(first, end, bad)
        with pytest.raises(ValueError):
            mirror_validate(first, end, bad)
    with pytest.raises(ValueError):                                   # a receipt for another range
        multi.validate_result(first, end - 1, r)


def test_production_surface_is_the_reference_module(ledger):
    _, production = ledger
    import psuedocubes_b200.production as P
    assert P.Frontier is production.Frontier
    assert P.load_production is production.load_production and P.save_compressed is production.save_compressed
