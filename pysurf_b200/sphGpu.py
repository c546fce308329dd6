"""The B200 backend of pySurf's SPH solver: ``PairSums`` over hand-written sm_100a CUDA.

This module is a drop-in for ``pysurf.sphGpu`` (src/pysurf/sphGpu.py:1482-2323): the same
class name, constructor, setters, host-step sums and device-resident steps, with the same
argument meanings, return shapes and errors, so ``WcsphSolver(config)`` with
``config.backend = 'gpu'`` drives it unchanged once ``pysurf_b200.install()`` has put it in
``pysurf.sphGpu``'s place.  Underneath, every call goes through the C-ABI of
``libpysurf_b200.so`` (include/pysurf_b200.h); there is no CPU path.

What it carries: the cubic spline and the Wendland C2 kernels; the plain and the limited
artificial viscosity; the continuity sum plain and corrected; the delta-SPH diffusive term in its
'molteni', 'hydrostatic' and 'antuono' forms; the extrapolated wall pressure; negative pressure;
the Shepard filter; XSPH; a periodic y axis; mixed smoothing lengths; container, bed and height
field enforcement; the delta-LES-SPH closure; particle shifting; the energy budget.

Beyond the reference's surface, ``advance`` runs a whole span of steps on the device with the
time step taken there (no host round trip per step), ``split`` refines on the device, and
``neighborList`` / ``cellOrderKey`` give the reference's neighbour rows and cell keys.
"""
from __future__ import annotations

import math

import numpy as np

from pysurf_b200 import _lib
from pysurf_b200._lib import check, dptr, f64, u8

maxGridCells = 2 ** 25
diffusionModes = {'none': 0, 'molteni': 1, 'hydrostatic': 2, 'antuono': 3}
# The energy budget's terms the device steps keep (src/pysurf/sphEnergy.py:88-98, deviceTerms)
energyTerms = ('pressureFluid', 'viscosityFluid', 'pressureWall', 'viscosityWall', 'gravityWork', 'continuityFluid',
               'continuityWall', 'correction', 'diffusion', 'floor', 'drift', 'clamp', 'shifting', 'filter')
taitExponent = 7.0


def cubicSplineNormalization(smoothingLength: float, dimensions: int) -> float:
    """The cubic spline's sigma: 10 / (7 pi h^2) in 2D, 1 / (pi h^3) in 3D."""
    h = smoothingLength
    return 10.0 / (7.0 * math.pi * h * h) if dimensions == 2 else 1.0 / (math.pi * h * h * h)


def wendlandNormalization(smoothingLength: float, dimensions: int) -> float:
    """The Wendland C2's sigma: 7 / (4 pi h^2) in 2D, 21 / (16 pi h^3) in 3D."""
    h = smoothingLength
    return 7.0 / (4.0 * math.pi * h * h) if dimensions == 2 else 21.0 / (16.0 * math.pi * h * h * h)


def kernelNormalization(kernelType: str, smoothingLength: float, dimensions: int) -> float:
    if kernelType == 'wendlandC2':
        return wendlandNormalization(smoothingLength, dimensions)
    return cubicSplineNormalization(smoothingLength, dimensions)


def gridDimensions(domainMin, domainMax, cellSize: float, dimensions: int) -> tuple:
    """Cells along x, y and z covering the domain, one support across (src/pysurf/sphGpu.py:1466-1478)."""
    extent = np.zeros(3)
    extent[:dimensions] = np.asarray(domainMax, dtype=float) - np.asarray(domainMin, dtype=float)
    cells = np.maximum(np.ceil(extent / cellSize).astype(int) + 3, 1)
    if dimensions == 2:
        cells[2] = 1
    while int(np.prod(cells)) > maxGridCells:
        cells = np.maximum((cells * 0.8).astype(int), 1)
    return tuple(int(count) for count in cells)


def padded(values) -> np.ndarray:
    """Vectors of 2 or 3 components as 3, the third zero for 2."""
    values = np.asarray(values, dtype=float)
    if values.shape[1] == 3:
        return np.ascontiguousarray(values)
    result = np.zeros((len(values), 3))
    result[:, :values.shape[1]] = values
    return result


def cellOrderKey(positions, cellWidth: float, shape, device: int = 0) -> np.ndarray:
    """``sphSolver.cellOrderKey`` (src/pysurf/sphSolver.py:1379-1408) on the device, bit-exact."""
    x = f64(positions)
    n, dim = x.shape
    keys = np.empty(n, dtype=np.int64)
    shp = np.array(list(shape) + [1] * (3 - len(shape)), dtype=np.int64)
    lib = _lib.load()
    check(lib.sph_cell_order_key(dptr(x), n, dim, float(cellWidth), shp.ctypes.data_as(_lib._pi64),
                                 keys.ctypes.data_as(_lib._pi64), int(device)), 'cellOrderKey')
    return keys


def _deviceIndex(device) -> int:
    if device is None:
        return 0
    if isinstance(device, int):
        return device
    text = str(device)
    if text.startswith('cuda'):
        return int(text.split(':')[1]) if ':' in text else 0
    raise ValueError(f"Device '{device}' is not a CUDA device; the B200 backend runs on CUDA only.")


def _checkDeviceTensor(tensor, shape, dtypes, device: int) -> None:
    """A contiguous CUDA tensor on `device` with the shape and one of the dtypes (names), or ValueError."""
    dtypes = (dtypes,) if isinstance(dtypes, str) else dtypes
    if not hasattr(tensor, 'data_ptr') or not getattr(tensor, 'is_cuda', False):
        raise ValueError('expected a CUDA tensor')
    if tensor.device.index != device:
        raise ValueError(f'expected a tensor on cuda:{device}, got {tensor.device}')
    if str(tensor.dtype).replace('torch.', '') not in dtypes:
        raise ValueError(f'expected dtype {" or ".join(dtypes)}, got {tensor.dtype}')
    if tuple(tensor.shape) != tuple(shape) or not tensor.is_contiguous():
        raise ValueError(f'expected a contiguous tensor of shape {tuple(shape)}, got {tuple(tensor.shape)}')


class PairSums:

    """

    The SPH pair sums and the time step of one particle system on a B200.

    For host steps, call `update` once per step, after the positions move, then any of the sums:
    every sum takes host arrays and returns a host array, float64, shaped as the compiled
    backend's.  For device steps, set the physics (`setPhysics`), copy the state up (`push`), set
    the boundary (`setBoundary`), call `residentRates` and `residentIntegrate` each step, or
    `advance` for a span of steps, and copy the state back (`pull`).

    Parameters are those of src/pysurf/sphGpu.py:1524-1569.

    """

    def __init__(self, dimensions: int, smoothingLength: float, domainMin, domainMax, period: float = 0.0,
                 separationPrecision: str = 'float64', device=None, kernelType: str = 'cubicSpline') -> None:
        if separationPrecision not in ('float64', 'float32'):
            raise ValueError(f"Separation precision '{separationPrecision}' is not 'float64' or 'float32'.")
        if kernelType not in ('cubicSpline', 'wendlandC2'):
            raise ValueError(f"Kernel '{kernelType}' is not 'cubicSpline' or 'wendlandC2'.")
        if period > 0.0 and dimensions != 3:
            raise ValueError('A periodic axis needs three dimensions: it is y.')
        self.dimensions = int(dimensions)
        self.smoothingLength = float(smoothingLength)
        self.kernelType = kernelType
        self.kind = 1 if kernelType == 'wendlandC2' else 0
        self.sigma = kernelNormalization(kernelType, smoothingLength, dimensions)
        self.sigmaUnit = kernelNormalization(kernelType, 1.0, dimensions)
        self.maxLength = self.smoothingLength
        self.minLength = self.smoothingLength
        self.uniformLengths = True
        self.period = float(period)
        self.precise = 1 if separationPrecision == 'float64' else 0
        self.device = _deviceIndex(device)
        self.count = 0
        self.physics: dict = {}
        self.diffusion = {'mode': 0, 'factor': 0.0, 'referenceDensity': 1000.0, 'gravityOverSound': 0.0}
        self.extrapolateWalls = False
        self.negativePressure = False
        self.correctContinuity = False
        self.limitViscosity = False
        self.trackEnergy = False
        self.shiftingEnabled = False
        self.closureEnabled = False
        self.compensatedSums = False
        self._lib = _lib.load()
        lower, upper = np.zeros(3), np.zeros(3)
        lower[:self.dimensions] = np.asarray(domainMin, dtype=float)[:self.dimensions]
        upper[:self.dimensions] = np.asarray(domainMax, dtype=float)[:self.dimensions]
        handle = _lib.C.c_void_p()
        check(self._lib.sph_create(self.dimensions, self.smoothingLength, dptr(lower), dptr(upper), self.period,
                                   self.precise, self.kind, self.device, _lib.C.byref(handle)), 'PairSums')
        self._handle = handle
        shape = np.zeros(3, dtype=np.int64)
        check(self._lib.sph_grid_shape(self._handle, shape.ctypes.data_as(_lib._pi64)))
        self.gridShape = tuple(int(c) for c in shape)
        self.cellsPerSupport = 3
        self._enforcement = None

    def __del__(self):
        handle = getattr(self, '_handle', None)
        if handle:
            try:
                self._lib.sph_destroy(handle)
            except Exception:
                pass
            self._handle = None

    # -- switches (src/pysurf/sphGpu.py:1701-1960) -- #
    @property
    def renormalizedDiffusion(self) -> bool:
        return self.diffusion['mode'] == diffusionModes['antuono']

    @property
    def needsCorrections(self) -> bool:
        return self.correctContinuity or self.renormalizedDiffusion

    @property
    def needsVelocityGradients(self) -> bool:
        return self.limitViscosity or self.closureEnabled

    def setContinuityCorrection(self, enabled: bool) -> None:
        self.correctContinuity = bool(enabled)
        check(self._lib.sph_set_continuity_correction(self._handle, int(self.correctContinuity)))

    def setViscosityLimiter(self, enabled: bool) -> None:
        self.limitViscosity = bool(enabled)
        check(self._lib.sph_set_viscosity_limiter(self._handle, int(self.limitViscosity)))

    def setClosure(self, enabled: bool, soundSpeed: float = 1.0, referenceDensity: float = 1000.0,
                   kinematicViscosity: float = 0.0) -> None:
        """Whether the accelerations and the diffusive term carry the delta-LES-SPH closure
        (src/pysurf/sphGpu.py:1752-1779; sphSolver.closureCoefficients, closureViscosity)."""
        check(self._lib.sph_set_closure(self._handle, int(bool(enabled)), float(soundSpeed), float(referenceDensity),
                                        float(kinematicViscosity)), 'setClosure')
        self.closureEnabled = bool(enabled)

    def setEnergyBudget(self, enabled: bool) -> None:
        """Whether the device steps keep the energy budget (src/pysurf/sphGpu.py:1780-1792): each fluid
        particle's running total of every term in `energyTerms`, from `push` to `energySums`."""
        check(self._lib.sph_set_energy_budget(self._handle, int(bool(enabled))), 'setEnergyBudget')
        self.trackEnergy = bool(enabled)

    def setCompensatedSums(self, enabled: bool) -> None:
        """Whether the momentum and continuity sums carry their running rounding error (Dot2
        compensation: each particle's du/dt and drho/dt as if summed in twice float32's precision;
        the terms stay float32).  Not with the energy budget."""
        check(self._lib.sph_set_compensated_sums(self._handle, int(bool(enabled))), 'setCompensatedSums')
        self.compensatedSums = bool(enabled)

    def energySums(self) -> np.ndarray:
        """Each term's energy over the device steps since `push` [J] (per unit depth in 2D), summed
        over the particles, in `energyTerms` order (src/pysurf/sphGpu.py:1805-1825).

        Raises ValueError while the budget is off."""
        if not self.trackEnergy:
            raise ValueError('The energy budget is off; see setEnergyBudget.')
        out = np.zeros(len(energyTerms))
        check(self._lib.sph_energy_sums(self._handle, dptr(out)), 'energySums')
        return out

    def fluidEnergy(self) -> np.ndarray:
        """The device state's fluid kinetic, potential and elastic energy [J] (per unit depth in 2D):
        the budget's terms sum to the change of their total."""
        out = np.zeros(3)
        check(self._lib.sph_fluid_energy(self._handle, dptr(out)), 'fluidEnergy')
        return out

    def setDiffusion(self, mode: str, delta: float, soundSpeed: float, referenceDensity: float, gravity: float) -> None:
        if mode not in diffusionModes:
            raise KeyError(mode)
        self.diffusion = {'mode': diffusionModes[mode], 'factor': 2.0 * delta * soundSpeed,
                          'referenceDensity': float(referenceDensity), 'gravityOverSound': gravity / soundSpeed ** 2}
        check(self._lib.sph_set_diffusion(self._handle, diffusionModes[mode], float(delta), float(soundSpeed),
                                          float(referenceDensity), float(gravity)), 'setDiffusion')

    def setWallPressure(self, extrapolated: bool) -> None:
        self.extrapolateWalls = bool(extrapolated)
        check(self._lib.sph_set_wall_pressure(self._handle, int(self.extrapolateWalls)))

    def setNegativePressure(self, enabled: bool) -> None:
        self.negativePressure = bool(enabled)
        check(self._lib.sph_set_negative_pressure(self._handle, int(self.negativePressure)))

    def setShifting(self, enabled: bool, mach: float = 0.1, spacing: float = 1.0, soundSpeed: float = 1.0,
                    local: bool = False) -> None:
        """Particle shifting (sphSolver.shiftingDisplacement) for every step that follows
        (src/pysurf/sphGpu.py:1927-1957): size CFL Ma (2h)^2, or 2 h |v_i| dt with `local`."""
        check(self._lib.sph_set_shifting(self._handle, int(bool(enabled)), float(mach), float(spacing),
                                         float(soundSpeed), int(bool(local))), 'setShifting')
        self.shiftingEnabled = bool(enabled)

    def setCellsPerSupport(self, cells: int) -> None:
        """Cells per kernel support of the device's cell list (1: 2h wide; 2: h wide; the default 3: 2h/3 wide)."""
        check(self._lib.sph_set_cells_per_support(self._handle, int(cells)))
        self.cellsPerSupport = int(cells)

    def setSweepOptions(self, neighborTable: bool = True, threadsPerParticle: int = 4) -> None:
        """Whether the sweeps read a per-step neighbour table (else they walk the cells; the sums are
        the same bits either way), and how many threads (1, 2, 4, 8) share each particle's neighbours."""
        check(self._lib.sph_set_sweep_options(self._handle, int(bool(neighborTable)), int(threadsPerParticle)),
              'setSweepOptions')

    # -- host steps (src/pysurf/sphGpu.py:1998-2113) -- #
    def _vectors(self, values) -> np.ndarray:
        return f64(values, (self.count, self.dimensions))

    def _scalars(self, values) -> np.ndarray:
        return f64(values, (self.count,))

    def update(self, positions, masses, isFluid, lengths=None) -> None:
        """Copy the positions, masses, fluid flags and smoothing lengths to the device and rebuild the cell list."""
        positions = f64(positions)
        count = len(positions)
        if count and positions.shape[1] != self.dimensions:
            raise ValueError(f'positions must have {self.dimensions} columns')
        masses = f64(np.broadcast_to(masses, (count,)))
        flags, flagPtr = u8(isFluid)
        lengthArray = None
        if lengths is not None:
            lengthArray = f64(lengths, (count,))
            longest = float(lengthArray.max()) if count else self.smoothingLength
            if count and longest > self.maxLength * (1.0 + 1e-9):
                raise ValueError(f'A smoothing length of {longest} m exceeds the {self.maxLength} m the hash '
                                 f'grid is built for.')
            self.minLength = float(lengthArray.min()) if count else self.smoothingLength
            # all equal exactly when the least is the greatest (a NaN makes both NaN, unequal)
            self.uniformLengths = self.minLength == longest if count else True
        else:
            self.minLength = self.smoothingLength
            self.uniformLengths = True
        self.count = count
        check(self._lib.sph_update(self._handle, count, dptr(positions), dptr(masses), flagPtr, dptr(lengthArray)),
              'update')

    def pairAccelerations(self, velocities, densities, pressures, soundSpeed: float, alpha: float,
                          boundaryViscosityFactor: float, gravity) -> np.ndarray:
        """Pressure gradient, artificial viscosity and gravity on the fluid, zero on the boundary [m/s^2]."""
        out = np.empty((self.count, self.dimensions))
        g = np.zeros(3)
        g[:self.dimensions] = np.asarray(gravity, dtype=float)[:self.dimensions]
        if self.count:
            check(self._lib.sph_pair_accelerations(self._handle, dptr(self._vectors(velocities)),
                                                   dptr(self._scalars(densities)), dptr(self._scalars(pressures)),
                                                   float(soundSpeed), float(alpha), float(boundaryViscosityFactor),
                                                   dptr(g), dptr(out)), 'pairAccelerations')
        return out

    def continuityRate(self, velocities, densities=None) -> np.ndarray:
        """d rho / dt for every particle, with the diffusive term `setDiffusion` set [kg/(m^3 s)]."""
        if (self.diffusion['mode'] != 0 or self.correctContinuity) and densities is None:
            raise ValueError('The diffusive term and the correction need the densities.')
        out = np.empty(self.count)
        if self.count:
            rho = None if densities is None else self._scalars(densities)
            check(self._lib.sph_continuity_rate(self._handle, dptr(self._vectors(velocities)), dptr(rho), dptr(out)),
                  'continuityRate')
        return out

    def xsphVelocity(self, velocities, densities, epsilon: float) -> np.ndarray:
        """The XSPH transport velocity of the fluid; boundary rows unchanged [m/s]."""
        out = np.empty((self.count, self.dimensions))
        if self.count:
            check(self._lib.sph_xsph_velocity(self._handle, dptr(self._vectors(velocities)),
                                              dptr(self._scalars(densities)), float(epsilon), dptr(out)),
                  'xsphVelocity')
        return out

    def wallPressure(self, densities, pressures, gravity, referenceDensity: float, soundSpeed: float) -> np.ndarray:
        """Every pressure with the boundary's taken from the fluid (`sphSolver.extrapolatedWallPressure`) [Pa]."""
        out = np.empty(self.count)
        g = np.zeros(3)
        g[:self.dimensions] = np.asarray(gravity, dtype=float)[:self.dimensions]
        if self.count:
            check(self._lib.sph_wall_pressure(self._handle, dptr(self._scalars(densities)),
                                              dptr(self._scalars(pressures)), dptr(g), float(referenceDensity),
                                              float(soundSpeed), dptr(out)), 'wallPressure')
        return out

    def shepardDensity(self, densities) -> np.ndarray:
        """The Shepard-filtered density of every particle [kg/m^3]."""
        out = np.empty(self.count)
        if self.count:
            check(self._lib.sph_shepard_density(self._handle, dptr(self._scalars(densities)), dptr(out)),
                  'shepardDensity')
        return out

    def velocityGradients(self, velocities, densities) -> np.ndarray:
        """G for every particle at the current positions, shape (N, dim, dim)."""
        if not self.needsVelocityGradients:
            raise ValueError('Neither the viscosity limiter nor the closure is on; see setViscosityLimiter, setClosure.')
        out = np.empty((self.count, self.dimensions, self.dimensions))
        if self.count:
            check(self._lib.sph_velocity_gradients(self._handle, dptr(self._vectors(velocities)),
                                                   dptr(self._scalars(densities)), dptr(out)), 'velocityGradients')
        return out

    def closureCoefficients(self, velocities, densities):
        """Each particle's alpha_i and delta_i at the current positions (sphSolver.closureCoefficients)."""
        if not self.closureEnabled:
            raise ValueError('The closure is off; see setClosure.')
        alphas, deltas = np.empty(self.count), np.empty(self.count)
        check(self._lib.sph_closure_coefficients(self._handle, dptr(f64(velocities)), dptr(f64(densities)),
                                                 dptr(alphas), dptr(deltas)), 'closureCoefficients')
        return alphas, deltas

    def correctionMatrices(self, densities) -> np.ndarray:
        """L for every particle at the current positions, shape (N, dim, dim)."""
        if not self.needsCorrections:
            raise ValueError('Neither the continuity correction nor the renormalized diffusion is on.')
        out = np.empty((self.count, self.dimensions, self.dimensions))
        if self.count:
            check(self._lib.sph_correction_matrices(self._handle, dptr(self._scalars(densities)), dptr(out)),
                  'correctionMatrices')
        return out

    def densityGradients(self, densities) -> np.ndarray:
        """Each particle's renormalized density gradient, shape (N, dim)."""
        if not self.renormalizedDiffusion:
            raise ValueError("The diffusive term is not 'antuono'; see setDiffusion.")
        out = np.empty((self.count, self.dimensions))
        if self.count:
            check(self._lib.sph_density_gradients(self._handle, dptr(self._scalars(densities)), dptr(out)),
                  'densityGradients')
        return out

    def shiftingDisplacement(self, densities, timeStep, velocities):
        """This step's shift, density change and velocity change of every particle, zero on the
        boundary and the free surface (src/pysurf/sphGpu.py:1980-1995)."""
        n, dim = self.count, self.dimensions
        shifts, velocityChanges, densityChanges = np.zeros((n, dim)), np.zeros((n, dim)), np.zeros(n)
        if n:
            check(self._lib.sph_shifting_displacement(self._handle, dptr(self._scalars(densities)), float(timeStep),
                                                      dptr(self._vectors(velocities)), dptr(shifts),
                                                      dptr(densityChanges), dptr(velocityChanges)),
                  'shiftingDisplacement')
        return shifts, densityChanges, velocityChanges

    def neighborList(self, radius: float | None = None) -> tuple:
        """Every particle's neighbours closer than `radius` (2h by default), itself excluded, as the
        reference's compressed rows (src/pysurf/sphCompiled.py:133-234), each row's set bit-exact."""
        radius = 2.0 * self.smoothingLength if radius is None else float(radius)
        offsets = np.zeros(self.count + 1, dtype=np.int64)
        total = _lib.C.c_int64(0)
        status = self._lib.sph_neighbor_list(self._handle, radius, offsets.ctypes.data_as(_lib._pi64), None, 0,
                                             _lib.C.byref(total))
        check(status, 'neighborList')
        neighbors = np.empty(max(total.value, 1), dtype=np.int32)
        check(self._lib.sph_neighbor_list(self._handle, radius, offsets.ctypes.data_as(_lib._pi64),
                                          neighbors.ctypes.data_as(_lib._pi32), len(neighbors), _lib.C.byref(total)),
              'neighborList')
        return offsets, neighbors[:total.value]

    # -- device steps (src/pysurf/sphGpu.py:2115-2323) -- #
    def canEnforce(self, boundary) -> bool:
        """Whether the device can enforce this boundary: none, a container, a bed or a height field."""
        return boundary is None or type(boundary).__name__ in ('ContainerBoundary', 'BedBoundary', 'HeightFieldBoundary')

    def setBoundary(self, boundary, particles) -> None:
        """The boundary the device steps enforce, as it stands: a piston holds its position and speed."""
        lib, handle = self._lib, self._handle
        kind = type(boundary).__name__ if boundary is not None else None
        if boundary is None:
            check(lib.sph_clear_boundary(handle))
        elif kind == 'ContainerBoundary':
            lower, upper = np.zeros(3), np.zeros(3)
            lower[:self.dimensions] = boundary.containerMin
            upper[:self.dimensions] = boundary.containerMax
            check(lib.sph_set_boundary_container(handle, dptr(lower), dptr(upper), int(bool(boundary.openTop))))
        elif kind == 'BedBoundary':
            bed, clearance = boundary.bathymetry, 0.25 * boundary.spacing
            mask = getattr(boundary, '_pistonMask', None)
            pistonSpeed = float(particles.velocities[mask, 0][0]) if mask is not None and mask.any() else 0.0
            sideWalls = boundary.width is not None and not boundary.periodic
            endLimit = bed.endX - clearance if boundary.endWallTop is not None else bed.endX
            bx, bz = f64(bed.x), f64(bed.z)
            check(lib.sph_set_boundary_bed(handle, dptr(bx), dptr(bz), len(bx), clearance, int(sideWalls),
                                           float(boundary.width or 0.0), int(boundary.wallTop is not None),
                                           float(boundary.wallX), pistonSpeed, float(endLimit)), 'setBoundary')
        elif kind == 'HeightFieldBoundary':
            field, clearance = boundary.field, 0.25 * boundary.spacing
            startX, endX, startY, endY = field.bounds
            table = f64(field.z)
            check(lib.sph_set_boundary_height_field(handle, dptr(table), table.shape[1], table.shape[0],
                                                    float(field.x[0]), float(field.y[0]), float(field.spacingX),
                                                    float(field.spacingY), clearance, startY + clearance,
                                                    endY - clearance, int(bool(boundary.offshoreWall)),
                                                    startX + clearance,
                                                    endX - clearance if boundary.endWall else endX), 'setBoundary')
        else:
            raise ValueError(f'The device cannot enforce a {type(boundary).__name__}; step from the host.')
        self._enforcement = kind

    def setPhysics(self, referenceDensity: float, soundSpeed: float, alpha: float, boundaryViscosityFactor: float,
                   gravity, xsphEpsilon: float, densityFloor: float) -> None:
        """The constants of the device step (src/pysurf/sphGpu.py:2173-2205)."""
        g = np.zeros(3)
        g[:self.dimensions] = np.asarray(gravity, dtype=float)[:self.dimensions]
        self.physics = {'referenceDensity': float(referenceDensity), 'soundSpeed': float(soundSpeed),
                        'stiffness': float(referenceDensity * soundSpeed ** 2 / taitExponent), 'alpha': float(alpha),
                        'boundaryViscosityFactor': float(boundaryViscosityFactor), 'gravity64': g[:self.dimensions],
                        'xsphEpsilon': float(xsphEpsilon), 'densityFloor': float(densityFloor)}
        check(self._lib.sph_set_physics(self._handle, float(referenceDensity), float(soundSpeed), float(alpha),
                                        float(boundaryViscosityFactor), dptr(g), float(xsphEpsilon),
                                        float(densityFloor)), 'setPhysics')

    def push(self, particles) -> None:
        """Copy a particle system's state to the device."""
        positions = f64(particles.positions)
        count = len(positions)
        lengths = getattr(particles, 'lengths', None)
        lengthArray = None if lengths is None else f64(lengths, (count,))
        # two passes over the lengths: all are equal exactly when the least is the greatest (a NaN
        # makes both NaN, which compare unequal, as an elementwise test would find)
        given = lengthArray is not None and count > 0
        longest = float(lengthArray.max()) if given else self.smoothingLength
        shortest = float(lengthArray.min()) if given else self.smoothingLength
        if given and longest > self.maxLength * (1.0 + 1e-9):
            raise ValueError(f'A smoothing length of {longest} m exceeds the {self.maxLength} m the hash '
                             f'grid is built for.')
        self.minLength = shortest
        self.uniformLengths = not given or shortest == longest
        flags, flagPtr = u8(particles.isFluid)
        self.count = count
        check(self._lib.sph_push(self._handle, count, dptr(positions), dptr(f64(particles.velocities)),
                                 dptr(f64(particles.densities)), dptr(f64(np.broadcast_to(particles.masses, (count,)))),
                                 flagPtr, dptr(lengthArray)), 'push')

    def pull(self, particles) -> None:
        """Copy the device state back into a particle system, in place."""
        if self.count == 0:
            return
        n, dim = self.count, self.dimensions
        shapes = {'positions': (n, dim), 'velocities': (n, dim), 'densities': (n,), 'pressures': (n,),
                  'accelerations': (n, dim)}
        targets = {}
        for name, shape in shapes.items():
            array = getattr(particles, name)
            # straight into the caller's array when it can take it (pinned arrays stay pinned)
            direct = (isinstance(array, np.ndarray) and array.dtype == np.float64 and array.shape == shape
                      and array.flags['C_CONTIGUOUS'] and array.flags['WRITEABLE'])
            targets[name] = array if direct else np.empty(shape)
        check(self._lib.sph_pull(self._handle, dptr(targets['positions']), dptr(targets['velocities']),
                                 dptr(targets['densities']), dptr(targets['pressures']),
                                 dptr(targets['accelerations']), None, None, None), 'pull')
        for name, value in targets.items():
            array = getattr(particles, name)
            if value is not array:
                array[:] = value

    # -- device arrays (torch CUDA tensors) in place of host arrays -- #

    def pushDevice(self, positions, velocities, densities, masses, isFluid, lengths=None) -> None:
        """`push` from device tensors on this handle's device: float64 positions and velocities (n, dim),
        densities and masses (n,), a uint8 or bool fluid flag (n,), and optionally the lengths (n,).
        The state is copied device to device; nothing crosses the host but the lengths' check."""
        n, dim = int(positions.shape[0]), self.dimensions
        shapes = ((positions, (n, dim)), (velocities, (n, dim)), (densities, (n,)), (masses, (n,)))
        for tensor, shape in shapes + (((lengths, (n,)),) if lengths is not None else ()):
            _checkDeviceTensor(tensor, shape, 'float64', self.device)
        _checkDeviceTensor(isFluid, (n,), ('uint8', 'bool'), self.device)
        if lengths is not None and n:
            longest = float(lengths.max())
            if longest > self.maxLength * (1.0 + 1e-9):
                raise ValueError(f'A smoothing length of {longest} m exceeds the {self.maxLength} m the hash '
                                 f'grid is built for.')
            self.minLength = float(lengths.min())
            self.uniformLengths = bool((lengths == lengths[0]).all())
        else:
            self.minLength, self.uniformLengths = self.smoothingLength, True
        self.count = n
        check(self._lib.sph_push_device(self._handle, n, positions.data_ptr(), velocities.data_ptr(),
                                        densities.data_ptr(), masses.data_ptr(), isFluid.data_ptr(),
                                        None if lengths is None else lengths.data_ptr()), 'pushDevice')

    def pullDevice(self, positions=None, velocities=None, densities=None, pressures=None, accelerations=None,
                   masses=None, lengths=None, isFluid=None) -> None:
        """`pull` into device tensors on this handle's device (float64, contiguous; isFluid uint8), any of
        them None.  Copied device to device; the tensors hold the state when this returns."""
        n, dim = self.count, self.dimensions
        vectors, scalars = (positions, velocities, accelerations), (densities, pressures, masses, lengths)
        for tensor in vectors:
            if tensor is not None:
                _checkDeviceTensor(tensor, (n, dim), 'float64', self.device)
        for tensor in scalars:
            if tensor is not None:
                _checkDeviceTensor(tensor, (n,), 'float64', self.device)
        if isFluid is not None:
            _checkDeviceTensor(isFluid, (n,), 'uint8', self.device)
        if n == 0:
            return
        ptr = lambda t: None if t is None else t.data_ptr()
        check(self._lib.sph_pull_device(self._handle, ptr(positions), ptr(velocities), ptr(densities), ptr(pressures),
                                        ptr(accelerations), ptr(masses), ptr(lengths), ptr(isFluid)), 'pullDevice')

    # -- the breaking tracker's reads (2D), on the device -- #

    def surfaceTops(self, x0: float, width: float, count: int, section=None) -> np.ndarray:
        """The highest fluid particle's height in each of `count` columns from x0 (-inf where empty).
        `section` (3D): (y, halfWidth), the fluid with |y_p - y| < halfWidth, its heights along z."""
        tops = np.empty(int(count))
        if section is None:
            check(self._lib.sph_surface_tops(self._handle, float(x0), float(width), int(count), dptr(tops)),
                  'surfaceTops')
        else:
            check(self._lib.sph_section_tops(self._handle, float(section[0]), float(section[1]), float(x0),
                                             float(width), int(count), dptr(tops)), 'surfaceTops')
        return tops

    def faceCells(self, lowX: float, highX: float, lowZ: float, half: float, start: float, base: float,
                  spacing: float, columns: int, bands: int, section=None) -> np.ndarray:
        """The face window's marked cells, (bands, columns) booleans (see sph_face_cells); `section` as
        in `surfaceTops`."""
        marks = np.empty((int(bands), int(columns)), dtype=np.uint8)
        window = (float(lowX), float(highX), float(lowZ), float(half), float(start), float(base), float(spacing),
                  int(columns), int(bands), marks.ctypes.data_as(_lib._pu8))
        if section is None:
            check(self._lib.sph_face_cells(self._handle, *window), 'faceCells')
        else:
            check(self._lib.sph_section_face_cells(self._handle, float(section[0]), float(section[1]), *window),
                  'faceCells')
        return marks.astype(bool)

    def bedSheet(self, bedX, bedZ, wetHeight: float, section=None) -> np.ndarray:
        """The x of the fluid particles less than `wetHeight` above the bed profile, in no set order;
        `section` as in `surfaceTops`."""
        bx, bz = f64(bedX), f64(bedZ)
        xs = np.empty(max(self.count, 1))
        found = _lib.C.c_int64(0)
        sheet = (dptr(bx), dptr(bz), len(bx), float(wetHeight), dptr(xs), len(xs), _lib.C.byref(found))
        if section is None:
            check(self._lib.sph_bed_sheet(self._handle, *sheet), 'bedSheet')
        else:
            check(self._lib.sph_section_bed_sheet(self._handle, float(section[0]), float(section[1]), *sheet),
                  'bedSheet')
        return xs[:found.value]

    def pullPositions(self, out: np.ndarray | None = None) -> np.ndarray:
        """The positions alone, in the caller's order (a tracker's read): into `out` when given."""
        n, dim = self.count, self.dimensions
        if out is None or out.shape != (n, dim) or out.dtype != np.float64 or not out.flags['C_CONTIGUOUS']:
            out = np.empty((n, dim))
        if n:
            check(self._lib.sph_pull(self._handle, dptr(out), None, None, None, None, None, None, None), 'pull')
        return out

    def residentRates(self, filterDensity: bool) -> tuple:
        """The first half of a device step; returns the largest fluid speed and acceleration."""
        speed, accel = _lib.C.c_double(0.0), _lib.C.c_double(0.0)
        check(self._lib.sph_resident_rates(self._handle, int(bool(filterDensity)), _lib.C.byref(speed),
                                           _lib.C.byref(accel)), 'residentRates')
        return float(speed.value), float(accel.value)

    def residentIntegrate(self, timeStep: float) -> None:
        """The second half of a device step: kick, continuity, density, XSPH, drift and enforcement."""
        check(self._lib.sph_resident_integrate(self._handle, float(timeStep)), 'residentIntegrate')

    def enforceBoundary(self) -> None:
        check(self._lib.sph_enforce_boundary(self._handle), 'enforceBoundary')

    def advance(self, time: float, step: int, untilTime: float, maxStep: int, shortestLength: float,
                cflNumber: float, maxTimeStep: float, filterInterval: int = 0, lastTimeStep: float = 0.0) -> tuple:
        """Steps on the device until `untilTime` or step `maxStep`, each step's dt taken there from its own
        maxima (src/pysurf/sphSolver.py:1941-1991, 1410-1424).  Returns (time, step, last dt)."""
        t, s, dt = _lib.C.c_double(time), _lib.C.c_int64(step), _lib.C.c_double(lastTimeStep)
        check(self._lib.sph_advance(self._handle, _lib.C.byref(t), _lib.C.byref(s), _lib.C.byref(dt),
                                    float(untilTime), int(maxStep), float(shortestLength), float(cflNumber),
                                    float(maxTimeStep), int(filterInterval)), 'advance')
        return float(t.value), int(s.value), float(dt.value)

    def neighborTableCapacity(self) -> int:
        """The neighbour table's row capacity now; 0 when the sweeps walk the cells."""
        cap = _lib.C.c_int64(0)
        check(self._lib.sph_neighbor_table(self._handle, _lib.C.byref(cap)))
        return int(cap.value)

    def setStream(self, stream) -> None:
        """The CUDA stream (a cudaStream_t as an int, e.g. torch.cuda.Stream().cuda_stream) the work goes on."""
        check(self._lib.sph_set_stream(self._handle, _lib.C.c_void_p(int(stream) if stream else 0)), 'setStream')

    def beginSteps(self, time: float, step: int, untilTime: float, maxStep: int, shortestLength: float,
                   cflNumber: float, maxTimeStep: float, filterInterval: int = 0, lastTimeStep: float = 0.0) -> None:
        """Set the device clock and limits for `enqueueSteps` (the three-call form of `advance`)."""
        check(self._lib.sph_begin_steps(self._handle, float(time), int(step), float(lastTimeStep), float(untilTime),
                                        int(maxStep), float(shortestLength), float(cflNumber), float(maxTimeStep),
                                        int(filterInterval)), 'beginSteps')

    def enqueueSteps(self, count: int) -> None:
        """Queue `count` device steps on the stream and return at once."""
        check(self._lib.sph_enqueue_steps(self._handle, int(count)), 'enqueueSteps')

    def finishSteps(self) -> tuple:
        """Wait for the queued steps; returns (time, step, last dt)."""
        t, s, dt = _lib.C.c_double(0.0), _lib.C.c_int64(0), _lib.C.c_double(0.0)
        check(self._lib.sph_finish_steps(self._handle, _lib.C.byref(t), _lib.C.byref(s), _lib.C.byref(dt)),
              'finishSteps')
        return float(t.value), int(s.value), float(dt.value)

    def stageNames(self) -> list:
        count = _lib.C.c_int64(0)
        self._lib.sph_stage_times(self._handle, None, 0, _lib.C.byref(count))
        return [self._lib.sph_stage_name(k).decode() for k in range(count.value)]

    def stageTimes(self) -> list:
        """Milliseconds of each stage of the last step that ran (device events inside its graph)."""
        count = _lib.C.c_int64(0)
        self._lib.sph_stage_times(self._handle, None, 0, _lib.C.byref(count))
        ms = np.zeros(count.value)
        check(self._lib.sph_stage_times(self._handle, dptr(ms), len(ms), _lib.C.byref(count)), 'stageTimes')
        return list(ms)

    def stepLaunches(self) -> int:
        """Kernels one device step launches."""
        count = _lib.C.c_int64(0)
        check(self._lib.sph_step_launches(self._handle, _lib.C.byref(count)), 'stepLaunches')
        return int(count.value)

    def lastAdvanceMilliseconds(self) -> float:
        ms = _lib.C.c_double(0.0)
        check(self._lib.sph_last_advance_ms(self._handle, _lib.C.byref(ms)))
        return float(ms.value)

    def split(self, mask, referenceDensity: float, lengthRatio: float = 1.0) -> int:
        """splitParticles (src/pysurf/sphRefinement.py:136-190) on the device-resident state."""
        flags, flagPtr = u8(mask)
        if len(flags) != self.count:
            raise ValueError('the mask must hold one flag per particle')
        count = _lib.C.c_int64(0)
        check(self._lib.sph_split(self._handle, flagPtr, float(referenceDensity), float(lengthRatio),
                                  _lib.C.byref(count)), 'split')
        total = _lib.C.c_int64(0)
        check(self._lib.sph_count(self._handle, _lib.C.byref(total)))
        self.count = int(total.value)
        return int(count.value)

    def merge(self, mask, referenceDensity: float, referenceMass: float, lengthRatio: float = 1.0):
        """mergeParticles (src/pysurf/sphRefinement.py:219-311) on the device-resident state: returns
        (groups, removed kinetic energy, source), source the caller index before the merge of each
        particle after."""
        flags, flagPtr = u8(mask)
        if len(flags) != self.count:
            raise ValueError('the mask must hold one flag per particle')
        groups, removed = _lib.C.c_int64(0), _lib.C.c_double(0.0)
        source = np.empty(max(self.count, 1), dtype=np.int64)
        check(self._lib.sph_merge(self._handle, flagPtr, float(referenceDensity), float(referenceMass),
                                  float(lengthRatio), _lib.C.byref(groups), _lib.C.byref(removed),
                                  source.ctypes.data_as(_lib._pi64)), 'merge')
        count = _lib.C.c_int64(0)
        check(self._lib.sph_count(self._handle, _lib.C.byref(count)))
        self.count = int(count.value)
        return int(groups.value), float(removed.value), source[:self.count]

    def splitCrestZone(self, x0: float, y0: float, width: float, nx: int, ny: int, threshold: float,
                       minMass: float, referenceDensity: float, lengthRatio: float = 0.5) -> int:
        """Split, on the device, every unsplit fluid particle (mass at least `minMass`) whose column
        (`width` across from (x0, y0), nx by ny) has its surface above `threshold`; returns how many."""
        count = _lib.C.c_int64(0)
        check(self._lib.sph_split_crest_zone(self._handle, float(x0), float(y0), float(width), int(nx), int(ny),
                                             float(threshold), float(minMass), float(referenceDensity),
                                             float(lengthRatio), _lib.C.byref(count)), 'splitCrestZone')
        total = _lib.C.c_int64(0)
        check(self._lib.sph_count(self._handle, _lib.C.byref(total)))
        self.count = int(total.value)
        return int(count.value)

    def frame(self) -> tuple:
        """The fluid particles' float32 positions (m, dim) and speeds (m,) from the device state, in the
        caller's order: the arrays of a run's frame (src/pysurf/sphFrames.py:60-100), without a float64 pull."""
        n, dim = self.count, self.dimensions
        positions, speeds = np.empty((n, dim), dtype=np.float32), np.empty(n, dtype=np.float32)
        flags = np.empty(n, dtype=np.uint8)
        if n:
            check(self._lib.sph_frame(self._handle, positions.ctypes.data_as(_lib._pf), speeds.ctypes.data_as(_lib._pf),
                                      flags.ctypes.data_as(_lib._pu8)), 'frame')
        fluid = flags.astype(bool)
        return positions[fluid], speeds[fluid]

    def pullState(self) -> dict:
        """The whole device state in the caller's order, masses, lengths and flags included."""
        n, dim = self.count, self.dimensions
        out = {'positions': np.empty((n, dim)), 'velocities': np.empty((n, dim)), 'densities': np.empty(n),
               'pressures': np.empty(n), 'accelerations': np.empty((n, dim)), 'masses': np.empty(n),
               'lengths': np.empty(n), 'isFluid': np.empty(n, dtype=np.uint8)}
        if n:
            check(self._lib.sph_pull(self._handle, dptr(out['positions']), dptr(out['velocities']),
                                     dptr(out['densities']), dptr(out['pressures']), dptr(out['accelerations']),
                                     dptr(out['masses']), dptr(out['lengths']),
                                     out['isFluid'].ctypes.data_as(_lib._pu8)), 'pull')
        out['isFluid'] = out['isFluid'].astype(bool)
        return out
