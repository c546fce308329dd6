"""Build the FP64 C oracle (test infrastructure) into oracle/_build/libsph_oracle.so.

The oracle is the parity checker for the CUDA backend; see sph_oracle.c's header.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SOURCE = os.path.join(HERE, 'sph_oracle.c')
LIBRARY = os.path.join(HERE, '_build', 'libsph_oracle.so')


def build(force: bool = False) -> str:
    """Compile the oracle when its source is newer than the library; returns the library path."""
    if not force and os.path.exists(LIBRARY) and os.path.getmtime(LIBRARY) >= os.path.getmtime(SOURCE):
        return LIBRARY
    os.makedirs(os.path.dirname(LIBRARY), exist_ok=True)
    # -ffp-contract=off keeps r^2 rounding term by term, as numba's neighbour test does
    subprocess.check_call(['gcc', '-O2', '-fopenmp', '-ffp-contract=off', '-shared', '-fPIC', '-Wall',
                           '-o', LIBRARY, SOURCE])
    return LIBRARY


if __name__ == '__main__':
    print(build(force=True))
