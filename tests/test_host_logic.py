"""Host-side logic of the drop-in that needs no GPU: argument checks, the install shim, case builders."""
import sys
import types

import numpy as np
import pytest

from conftest import golden
from pysurf_b200 import cases, sphGpu


def test_constructor_rejects_what_the_reference_rejects():
    # src/pysurf/sphGpu.py:1527-1532: these raise before any device work
    with pytest.raises(ValueError):
        sphGpu.PairSums(2, 0.1, [0, 0], [1, 1], separationPrecision='float16')
    with pytest.raises(ValueError):
        sphGpu.PairSums(2, 0.1, [0, 0], [1, 1], kernelType='quintic')
    with pytest.raises(ValueError):
        sphGpu.PairSums(2, 0.1, [0, 0], [1, 1], period=1.0)
    with pytest.raises(ValueError):
        sphGpu.PairSums(2, 0.1, [0, 0], [1, 1], device='cpu')


def test_grid_dimensions_follow_the_reference():
    # src/pysurf/sphGpu.py:1466-1478
    assert sphGpu.gridDimensions([0, 0], [4, 3], 0.052, 2) == (80, 61, 1)
    assert sphGpu.gridDimensions([0, 0, 0], [1, 1, 1], 0.5, 3) == (5, 5, 5)


def test_install_puts_the_backend_in_pysurfs_place():
    fakePysurf = types.ModuleType('pysurf')
    fakeSolver = types.ModuleType('pysurf.sphSolver')

    class WcsphSolver:
        def advance(self, untilTime, maxSteps=None):
            return 'reference'
    fakeSolver.WcsphSolver = WcsphSolver
    fakePysurf.sphSolver = fakeSolver
    saved = {k: sys.modules.get(k) for k in ('pysurf', 'pysurf.sphSolver', 'pysurf.sphGpu')}
    sys.modules['pysurf'] = fakePysurf
    sys.modules['pysurf.sphSolver'] = fakeSolver
    try:
        import pysurf_b200
        pysurf_b200.install()
        assert sys.modules['pysurf.sphGpu'] is sphGpu
        assert fakePysurf.sphGpu is sphGpu
        assert getattr(WcsphSolver.advance, '_b200', False)
        # a solver without the B200 backend keeps the reference's loop
        solver = WcsphSolver()
        solver._gpu, solver._boundary, solver._energy = None, None, None
        assert solver.advance(1.0) == 'reference'
        pysurf_b200.install()      # idempotent
        assert getattr(WcsphSolver.advance, '_b200', False)
    finally:
        for key, value in saved.items():
            if value is None:
                sys.modules.pop(key, None)
            else:
                sys.modules[key] = value


def test_the_beach_start_is_the_references():
    g = golden('beach.npz', 'beach')
    case = cases.solitaryBeach(particlesPerDepth=8)
    s = case.state
    assert s.positions.shape == g['positions'].shape
    assert np.allclose(s.positions, g['positions'], rtol=0.0, atol=1e-12)
    assert np.allclose(s.velocities, g['velocities'], rtol=0.0, atol=1e-12)
    assert np.array_equal(s.isFluid, g['isFluid'])
    assert np.allclose(s.masses, g['masses'], rtol=1e-15)
    assert np.allclose(s.densities, g['densities'], rtol=1e-14)


def test_the_dam_break_tank_is_the_references():
    g = golden('beach.npz', 'dam')
    assert np.allclose(cases.containerPositions([0, 0], [4, 3], 0.1, 3, True), g['boundary'], atol=1e-12)
    assert np.allclose(cases.latticePoints([0, 0], [1, 2], 0.1), g['column'], atol=1e-12)
    case = cases.damBreak()
    assert case.fluidCount == 5000


def test_the_benchmark_beach_size():
    case = cases.solitaryBeach(particlesPerDepth=64)
    # tens of thousands of fluid particles per 10 depths of flat water at 64 ppd
    assert 90_000 < case.fluidCount < 130_000
    assert case.smoothingLength == pytest.approx(3.0 / 64)
