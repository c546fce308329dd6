"""Compile the CUDA backend for sm_100a into pysurf_b200/libpysurf_b200.so (in-tree).

    python -m pysurf_b200.build          # rebuild when a source is newer than the library

nvcc cross-compiles without a GPU, so this runs on any machine with the CUDA toolkit.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIBRARY = os.path.join(HERE, 'libpysurf_b200.so')
SOURCES = ['csrc/sph_kernels.cu', 'csrc/sph_sweep_kernels.cu', 'csrc/sph_system.cu', 'csrc/sph_noalloc.cu',
           'csrc/sph_surface.cu', 'csrc/sph_merge.cu']
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC', '-shared']


def inputs() -> list:
    files = [os.path.join(HERE, s) for s in SOURCES]
    files += glob.glob(os.path.join(HERE, 'csrc', '*.cuh')) + glob.glob(os.path.join(HERE, 'csrc', '*.h'))
    files.append(os.path.join(ROOT, 'include', 'pysurf_b200.h'))
    return files


def stale() -> bool:
    if not os.path.exists(LIBRARY):
        return True
    built = os.path.getmtime(LIBRARY)
    return any(os.path.getmtime(f) > built for f in inputs())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return LIBRARY
    nvcc = os.environ.get('NVCC', 'nvcc')
    command = [nvcc] + ARCH + FLAGS + ['-o', LIBRARY] + [os.path.join(HERE, s) for s in SOURCES]
    if verbose:
        print(' '.join(command))
    subprocess.check_call(command, cwd=HERE)
    return LIBRARY


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose=True))
