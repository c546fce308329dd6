"""The reference's own solver driving this backend through the drop-in boundary.

pySurf is installed unmodified under baseline/_ref (pip install --no-deps of the reference; its plotting
and unit libraries are absent here, so the package object, ``pysurf.constants`` and ``pysurf.figures``
are stubbed as its own test suite's imports need, src/pysurf/constants.py:29-38).  ``pysurf_b200.install()``
puts ``PairSums`` in ``pysurf.sphGpu``'s place, and the reference's ``WcsphSolver`` with
``config.backend = 'gpu'`` then constructs, configures and steps it exactly as it would its Warp backend
(src/pysurf/sphSolver.py:1499-1518, 1527-1605, 1700-1724, 1941-1991):

* host steps (``solver.step``), against the reference's compiled (numba) backend on its sloshing tank,
  at its own GPU test's tolerances (tests/testSphGpu.py:417-438);
* device-resident spans (``solver.advance``) of the deltaSph options, against its numpy backend, at the
  tolerances it holds its float32 device to against numpy (tests/testSphGpu.py:503-517).
"""
import math
import os
import sys
import types

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

REFERENCE = os.path.join(ROOT, 'baseline', '_ref')


@pytest.fixture
def reference():
    """The reference package from baseline/_ref under stub constants and figures, with this backend
    installed; sys.modules is restored afterwards."""
    if not os.path.isfile(os.path.join(REFERENCE, 'pysurf', 'sphSolver.py')):
        pytest.skip('the reference is not installed under baseline/_ref')
    saved = {name: module for name, module in sys.modules.items() if name == 'pysurf' or name.startswith('pysurf.')}
    for name in saved:
        del sys.modules[name]
    package = types.ModuleType('pysurf')
    package.__path__ = [os.path.join(REFERENCE, 'pysurf')]
    constants = types.ModuleType('pysurf.constants')
    constants.gravity = 9.80665
    constants.freshwaterDensity = 998.2
    constants.freshwaterKinematicViscosity = 1.0034e-6
    constants.seawaterDensity = 1025.0
    figures = types.ModuleType('pysurf.figures')
    sys.modules.update({'pysurf': package, 'pysurf.constants': constants, 'pysurf.figures': figures})
    package.constants, package.figures = constants, figures
    import pysurf_b200
    pysurf_b200.install()
    yield package
    for name in [n for n in sys.modules if n == 'pysurf' or n.startswith('pysurf.')]:
        del sys.modules[name]
    sys.modules.update(saved)


def sloshing(backend, **options):
    from pysurf.sphSolver import WcsphSolver
    from pysurf.WaterSim.scenarios.sloshingTank import SloshingTankConfig, createSloshingTank
    tank = SloshingTankConfig(tankWidth=0.2, tankHeight=0.15, fillRatio=0.5, initialTiltDeg=10.0,
                              particleSpacing=0.005)
    config, particles, boundary = createSloshingTank(tank)
    config.backend = backend
    for name, value in options.items():
        setattr(config, name, value)
    solver = WcsphSolver(config, boundary=boundary)
    solver.initialize(particles)
    return solver, particles


def test_the_reference_solver_steps_this_backend_as_its_compiled_one(reference):
    pytest.importorskip('numba')
    from pysurf_b200.sphGpu import PairSums
    states = []
    for backend in ('compiled', 'gpu'):
        solver, particles = sloshing(backend)
        if backend == 'gpu':
            assert isinstance(solver._gpu, PairSums)
        for _ in range(60):
            solver.step()
        states.append((particles.positions.copy(), particles.velocities.copy(), solver.time))
    assert states[1][2] == pytest.approx(states[0][2], rel=1e-5)
    assert np.abs(states[1][0] - states[0][0]).max() <= 1e-7
    assert np.abs(states[1][1] - states[0][1]).max() <= 1e-4


def test_the_reference_solver_advances_this_backend_on_the_device(reference):
    from pysurf_b200.sphGpu import PairSums
    delta = dict(densityDiffusion='hydrostatic', densityFilterInterval=0, xsphEpsilon=0.0,
                 wallPressure='extrapolated', continuityCorrection=True, densityFloor=0.9, viscosityLimiter=True,
                 maxTimeStep=1e-3)
    states = []
    for backend in ('numpy', 'gpu'):
        solver, particles = sloshing(backend, **delta)
        if backend == 'gpu':
            assert isinstance(solver._gpu, PairSums) and solver._gpu.canEnforce(solver._boundary)
        state = solver.advance(math.inf, 40)
        assert solver._step == 40
        states.append((particles.positions.copy(), particles.velocities.copy(), particles.densities.copy(),
                       solver.time))
    (x0, v0, r0, t0), (x1, v1, r1, t1) = states
    assert t1 == pytest.approx(t0, rel=1e-4)
    assert np.abs(x1 - x0).max() < 1e-6
    assert np.abs(v1 - v0).max() < 1e-3
    assert np.abs(r1 - r0).max() < 1e-3
