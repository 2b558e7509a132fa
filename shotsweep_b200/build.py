"""Build libshotsweep.so (sm_100a) in-tree with nvcc.

    python -m shotsweep_b200.build [--verbose]

The library lands next to this file so that it travels with the source tree.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
SOURCES = sorted((HERE / 'csrc').glob('*.cu'))
HEADERS = [ROOT / 'include' / 'shotsweep.h', *sorted((HERE / 'csrc').glob('*.h')), *sorted((HERE / 'csrc').glob('*.cuh'))]
LIBRARY = HERE / 'libshotsweep.so'
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']


def nvcc():
    path = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    if not Path(path).exists():
        raise RuntimeError('nvcc not found; the CUDA toolkit is required to build libshotsweep')
    return path


def command(output=LIBRARY, verbose=False, extra=()):
    cmd = [nvcc(), *ARCH, '-O3', '-lineinfo', '-std=c++17', '-ftz=false',
           '-Xcompiler', '-fPIC', '-shared', f'-I{ROOT / "include"}', '-o', str(output),
           *[str(s) for s in SOURCES], '-lcudart', *extra]
    if verbose:
        cmd.insert(1, '-Xptxas=-v')
    return cmd


def stale(output=LIBRARY):
    if not output.exists():
        return True
    t = output.stat().st_mtime
    return any(p.stat().st_mtime > t for p in SOURCES + HEADERS)


def build(force=False, verbose=False, output=LIBRARY):
    """Compile the library if it is missing or older than its sources."""
    if not force and not stale(output):
        return output
    tmp = output.with_suffix('.so.tmp')
    cmd = command(tmp, verbose)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError('nvcc failed:\n' + ' '.join(cmd) + '\n' + res.stdout + res.stderr)
    if verbose:
        sys.stderr.write(res.stdout + res.stderr)
    os.replace(tmp, output)
    return output


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('--verbose', action='store_true')
    ap.add_argument('--force', action='store_true')
    a = ap.parse_args()
    print(build(force=a.force or a.verbose, verbose=a.verbose))
