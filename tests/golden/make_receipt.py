"""Write golden_lease_receipt.json: this library's compact receipt of the reference's golden lease.

Run from the repository root on a machine with a B200 (the receipt comes from the device path):

    python tests/golden/make_receipt.py [output path]

The receipt is optimized.compute_lease over [575222931200000000, 575224569600000000) at p = 619,
as a worker hands it to the reference's ledger (SharedFrontier.complete, Frontier.complete).
Its timing fields are the ones measured in the run that wrote it; the tests compare every other
field.  tests/test_ledger.py commits it through the reference's unchanged ledger code, and
tests/test_gpu_parity.py checks that the device path still produces it.
"""
from __future__ import annotations

import json
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))


def main(out: Path) -> None:
    from psuedocubes_b200.batch_experiment import MaskedMatcher
    from psuedocubes_b200.focus import A619, B619, Config
    from psuedocubes_b200.gpu import GPUFocus, Runtime
    from psuedocubes_b200.optimized import compute_lease
    gold = json.loads((HERE / 'golden_lease.json').read_text())
    runtime = Runtime(time.monotonic() + 600, 8 * 1024**3)
    config = Config(619, 10**27, 3 * 10**27, A619, B619)
    af, bf = (GPUFocus(runtime, f) for f in config.focuses())
    receipt = compute_lease(MaskedMatcher(runtime, config), af, bf, int(gold['first']), int(gold['end']))
    if receipt['subtile_scopes'][0]['transcript_sha256'] != gold['transcript_sha256']:
        raise ArithmeticError('the device path no longer reproduces the golden lease')
    out.write_text(json.dumps(dict(first=gold['first'], end=gold['end'], receipt=receipt), indent=1,
                              sort_keys=True) + '\n')
    print('wrote', out)
    runtime.close()


if __name__ == '__main__':
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else HERE / 'golden_lease_receipt.json')
