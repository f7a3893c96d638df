"""Build libpcube.so in-tree for sm_100a with nvcc (no JIT, no torch extension cache)."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / 'csrc'
OUT = HERE / '_lib' / 'libpcube.so'
SOURCES = ('runtime.cu', 'wheel.cu', 'sieve.cu', 'receipt.cu', 'cubes.cu')
FLAGS = ['-gencode', 'arch=compute_100a,code=sm_100a', '-lineinfo', '-O3', '-std=c++17',
         '-Xcompiler', '-fPIC', '-shared', '--expt-relaxed-constexpr']


def nvcc() -> str:
    found = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    if not Path(found).exists():
        raise RuntimeError('nvcc not found')
    return found


def stale() -> bool:
    if not OUT.exists():
        return True
    mtime = OUT.stat().st_mtime
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob('*.cuh')) + [HERE.parent / 'include' / 'pcube.h']
    return any(p.stat().st_mtime > mtime for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the CUDA sources into psuedocubes_b200/_lib/libpcube.so (skipped when current)."""
    if not force and not stale():
        return OUT
    OUT.parent.mkdir(parents=True, exist_ok=True)
    tmp = OUT.with_suffix('.so.tmp')
    cmd = [nvcc(), *FLAGS, *(['-Xptxas', '-v'] if verbose else []), '-o', str(tmp),
           *[str(CSRC / s) for s in SOURCES]]
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode:
        sys.stderr.write(result.stdout + result.stderr)
        raise RuntimeError('nvcc failed building libpcube')
    if verbose:
        sys.stderr.write(result.stderr)
    os.replace(tmp, OUT)
    return OUT


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose='-v' in sys.argv))
