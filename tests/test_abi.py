"""The C-ABI library loads and exports every entry point include/pysurf_b200.h declares (no GPU needed)."""
import os
import re
import subprocess

from conftest import ROOT

HEADER = os.path.join(ROOT, 'include', 'pysurf_b200.h')


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r'^\s*(?:int|const char \*)\s*(sph_\w+)\s*\(', text, flags=re.M)))


def test_header_declares_the_reference_interface():
    names = declared()
    # one entry point per PairSums method the solver calls (src/pysurf/sphGpu.py:1998-2323)
    for name in ('sph_update', 'sph_pair_accelerations', 'sph_continuity_rate', 'sph_xsph_velocity',
                 'sph_wall_pressure', 'sph_shepard_density', 'sph_push', 'sph_pull', 'sph_resident_rates',
                 'sph_resident_integrate', 'sph_enforce_boundary', 'sph_set_physics', 'sph_set_diffusion'):
        assert name in names


def test_library_exports_every_declared_symbol():
    from pysurf_b200 import _lib
    lib = _lib.load()
    names = declared()
    for name in names:
        assert hasattr(lib, name), name
    # and the binding knows every one of them
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)
    nm = subprocess.run(['nm', '-D', '--defined-only', _lib.LIBRARY], capture_output=True, text=True).stdout
    exported = set(re.findall(r' T (sph_\w+)', nm))
    assert set(names) <= exported


def test_library_is_built_for_sm_100a():
    # the one architecture the build passes nvcc; on a GPU, tests/test_gpu_device_arrays.py asks the
    # CUDA runtime which architecture the loaded kernels carry
    from pysurf_b200 import build
    assert build.ARCH == ['-gencode', 'arch=compute_100a,code=sm_100a']
    assert not any(flag.startswith(('-arch', '--gpu-architecture', '-gencode')) for flag in build.FLAGS)
