"""Plain containers for a particle system and the boundaries the device enforces.

They carry the attribute names of the reference's own classes (``pysurf.sphParticles.ParticleSystem``,
src/pysurf/sphParticles.py:41-124; ``ContainerBoundary``, ``BedBoundary``, ``HeightFieldBoundary``,
src/pysurf/sphBoundaries.py:61-640), so ``PairSums.push``/``pull``/``setBoundary`` take either the
reference's objects or these.  They hold data only: seeding and host-side enforcement stay with
the reference, and the tests and benchmarks here build their inputs with ``pysurf_b200.cases``.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class ParticleState:
    """SoA particle state, fluid first then boundary, vectors (N, dim), scalars (N,)."""
    positions: np.ndarray
    velocities: np.ndarray
    accelerations: np.ndarray
    densities: np.ndarray
    pressures: np.ndarray
    masses: np.ndarray
    isFluid: np.ndarray
    lengths: np.ndarray | None = None

    @classmethod
    def assemble(cls, fluidPositions, boundaryPositions, spacing: float, referenceDensity: float,
                 fluidVelocities=None) -> 'ParticleState':
        """Fluid and boundary positions of a lattice of the given spacing, each particle rho0 s^dim
        (src/pysurf/sphParticles.py:81-124)."""
        fluid = np.asarray(fluidPositions, dtype=float)
        wall = np.asarray(boundaryPositions, dtype=float).reshape(-1, fluid.shape[1])
        nf, nb, dim = len(fluid), len(wall), fluid.shape[1]
        velocities = np.zeros((nf + nb, dim))
        if fluidVelocities is not None:
            velocities[:nf] = fluidVelocities
        return cls(positions=np.vstack([fluid, wall]), velocities=velocities, accelerations=np.zeros((nf + nb, dim)),
                   densities=np.full(nf + nb, referenceDensity), pressures=np.zeros(nf + nb),
                   masses=np.full(nf + nb, referenceDensity * spacing ** dim),
                   isFluid=np.concatenate([np.ones(nf, dtype=bool), np.zeros(nb, dtype=bool)]))

    @property
    def nParticles(self) -> int:
        return len(self.positions)

    @property
    def dimensions(self) -> int:
        return self.positions.shape[1]

    def copy(self) -> 'ParticleState':
        return ParticleState(**{k: (None if v is None else np.array(v, copy=True)) for k, v in self.__dict__.items()})


@dataclass
class ContainerBoundary:
    containerMin: np.ndarray
    containerMax: np.ndarray
    spacing: float
    nLayers: int = 3
    openTop: bool = True

    @property
    def dimensions(self) -> int:
        return len(self.containerMin)


@dataclass
class Profile:
    """A bed profile: vertices (x, z), x strictly increasing (src/pysurf/bathymetry.py:66-230)."""
    x: np.ndarray
    z: np.ndarray
    stillWaterLevel: float = 0.0

    @property
    def startX(self) -> float:
        return float(self.x[0])

    @property
    def endX(self) -> float:
        return float(self.x[-1])

    def elevation(self, x):
        return np.interp(x, self.x, self.z)

    def depth(self, x):
        """Still water depth max(0, swl - z_b(x)) (src/pysurf/bathymetry.py:227-231)."""
        return np.maximum(0.0, self.stillWaterLevel - self.elevation(x))


@dataclass
class BedBoundary:
    bathymetry: Profile
    spacing: float
    nLayers: int = 3
    wallTop: float | None = None
    width: float | None = None
    endWallTop: float | None = None
    periodic: bool = False
    wallX: float = 0.0
    _pistonMask: np.ndarray | None = None


@dataclass
class HeightTable:
    """A height field: z (ny, nx) on grid x (nx,), y (ny,), and the tank's bounds."""
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    bounds: tuple
    stillWaterLevel: float = 0.0

    @property
    def spacingX(self) -> float:
        return float(self.x[1] - self.x[0])

    @property
    def spacingY(self) -> float:
        return float(self.y[1] - self.y[0])


@dataclass
class HeightFieldBoundary:
    field: HeightTable
    spacing: float
    nLayers: int = 3
    wallTop: float = 1.0
    offshoreWall: bool = True
    endWall: bool = True
