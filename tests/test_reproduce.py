"""The bounded reproduction command (tools/reproduce.py:20-61): its argument and environment checks
on the host, and one run on the device with --compare-baseline against the plain per-tile matcher."""
from __future__ import annotations

import json

import pytest

from psuedocubes_b200 import reproduce
from psuedocubes_b200.focus import B619


def test_refusals_before_any_device_use(tmp_path, monkeypatch):
    out = tmp_path / 'record.json'
    monkeypatch.setenv('CUDA_VISIBLE_DEVICES', '0')
    for argv in (['--batches', '0'], ['--batches', '257'], ['--first', str(B619)], ['--first', '-1']):
        with pytest.raises(ValueError, match='bounded canonical scope'):
            reproduce.main(argv + ['--output', str(out)])
    out.write_text('{}')
    with pytest.raises(ValueError, match='new output path'):
        reproduce.main(['--output', str(out)])
    out.unlink()
    for visible in ('', '0,1'):
        monkeypatch.setenv('CUDA_VISIBLE_DEVICES', visible)
        with pytest.raises(ValueError, match='one available GPU'):
            reproduce.main(['--output', str(out)])
    assert not out.exists()


@pytest.mark.gpu
def test_two_golden_batches_with_the_plain_baseline(tmp_path, monkeypatch, capsys):
    monkeypatch.setenv('CUDA_VISIBLE_DEVICES', '0')
    out = tmp_path / 'record.json'
    record = reproduce.main(['--first', '575222931200000000', '--batches', '2', '--compare-baseline',
                             '--output', str(out)])
    assert record['status'] == 'PASS' and record['baseline_compared'] and record['production_coverage'] == 0
    assert record['end'] == str(575222931200000000 + 2 * 6_400_000_000)
    assert json.loads(out.read_text())['result']['subtile_scopes'] == record['result']['subtile_scopes']
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line['status'] == 'PASS' and line['candidates'] == record['result']['valid_focused_candidates']
