"""pysurf_b200 -- a B200 (sm_100a) backend for pySurf's weakly compressible delta-SPH step.

    from pysurf_b200.sphGpu import PairSums      # the drop-in for pysurf.sphGpu.PairSums
    import pysurf_b200; pysurf_b200.install()    # make WcsphSolver(backend='gpu') use it

The sums, the cell list, the integrator and the boundary enforcement are CUDA kernels in
pysurf_b200/csrc, compiled into libpysurf_b200.so (``python -m pysurf_b200.build``) and reached
through the C-ABI in include/pysurf_b200.h.
"""
from __future__ import annotations

import sys

__all__ = ['install', 'PairSums']


def __getattr__(name):
    if name == 'PairSums':
        from pysurf_b200.sphGpu import PairSums
        return PairSums
    raise AttributeError(name)


def install(fastAdvance: bool = True) -> None:
    """Put this backend in ``pysurf.sphGpu``'s place, so ``config.backend = 'gpu'`` runs on it.

    With ``fastAdvance``, ``WcsphSolver.advance`` runs each span of device steps in one call to the
    device (``PairSums.advance``), the time step taken there; the state, clock and results are those
    of the reference's loop (src/pysurf/sphSolver.py:1941-1991).  pySurf must be importable.
    """
    import pysurf
    from pysurf_b200 import sphGpu
    sys.modules['pysurf.sphGpu'] = sphGpu
    pysurf.sphGpu = sphGpu
    if not fastAdvance:
        return
    from pysurf import sphSolver
    solver = sphSolver.WcsphSolver
    if getattr(solver.advance, '_b200', False):
        return
    original = solver.advance

    def advance(self, untilTime: float, maxSteps: int | None = None):
        gpu = self._gpu
        if not isinstance(gpu, sphGpu.PairSums) or not gpu.canEnforce(self._boundary) or self._energy is not None:
            return original(self, untilTime, maxSteps)
        config, p = self._config, self._particles
        lastStep = self._step + maxSteps if maxSteps is not None else 2 ** 62
        if not (self._time < untilTime and self._step < lastStep):
            return self.currentState
        gpu.setPhysics(config.referenceDensity, self._speedOfSound, config.alphaViscosity,
                       config.boundaryViscosityFactor, config.gravity, config.xsphEpsilon,
                       config.densityFloor * config.referenceDensity)
        gpu.push(p)
        gpu.setBoundary(self._boundary, p)
        self._time, self._step, self._dt = gpu.advance(self._time, self._step, untilTime, lastStep,
                                                       self.shortestLength, config.cflNumber, config.maxTimeStep,
                                                       config.densityFilterInterval, self._dt)
        gpu.pull(p)
        return self.currentState

    advance._b200 = True
    advance.__doc__ = original.__doc__
    solver.advance = advance
