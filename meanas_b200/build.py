"""Build recipe for ``libmeanas_fdfd.so`` (sm_100a), written next to this file.

``python -m meanas_b200.build`` compiles ``csrc/fdfd_lib.cu`` with nvcc for
``sm_100a`` into ``meanas_b200/libmeanas_fdfd.so``.  The library is built in-tree
so it travels with the source tree; nothing is installed.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / 'libmeanas_fdfd.so'
SOURCES = [HERE / 'csrc' / 'fdfd_lib.cu']
DEPS = SOURCES + [HERE / 'csrc' / 'fdfd_device.cuh', HERE / 'csrc' / 'fdfd_ops.cuh', HERE / 'csrc' / 'fdfd_csr.cuh', HERE / 'csrc' / 'fdfd_fdtd.cuh',
                  HERE.parent / 'include' / 'meanas_fdfd.h']
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']


def nvcc() -> str:
    for cand in (os.environ.get('NVCC'), '/usr/local/cuda/bin/nvcc', 'nvcc'):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return 'nvcc'


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in DEPS if p.exists())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build():
        return LIB
    cmd = [nvcc(), *ARCH, '-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC', '-shared',
           '-o', str(LIB), *map(str, SOURCES)]
    if verbose:
        cmd.insert(-len(SOURCES), '-Xptxas=-v')
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose='-v' in sys.argv)
    print(LIB)
