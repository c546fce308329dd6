"""Workload builders: the benchmark cases laid out as the reference lays them out.

Set-up only (nothing here runs per step).  Each builder restates the reference's seeding so the
benchmarks and GPU tests run without it; tests/test_cases.py checks them against starts the
reference itself built (tests/golden/beach.npz).

    damBreak            a 1 x 2 m column in a 4 x 3 m tank, 3 wall layers, jittered lattice
    solitaryBeach       a first-order solitary wave over a plane beach, the deltaSph scheme
                        (src/pysurf/BreakingWave.py:658-760 with src/pysurf/waveMakers.py:282-329)
    ridgeWave3D         a solitary wave crossing a Gaussian ridge at 25 degrees in a walled 3D tank
                        (src/pysurf/BreakingWave3D.py:630-700, src/pysurf/sphBoundaries.py:498-595)

Each returns a ``Case``: the particle state, the boundary, and the solver configuration the
reference's ``SimulationConfig``/``WcsphSolver`` would hold for it.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from pysurf_b200.state import BedBoundary, ContainerBoundary, HeightFieldBoundary, HeightTable, ParticleState, Profile

GRAVITY = 9.80665            # src/pysurf/constants.py:29
FRESHWATER = 998.2           # src/pysurf/constants.py:33


@dataclass
class Case:
    """A particle system, its boundary and the scheme it runs (the fields of SimulationConfig it uses)."""
    name: str
    state: ParticleState
    boundary: object
    dimensions: int
    spacing: float
    smoothingLength: float
    kernelType: str
    domainMin: np.ndarray
    domainMax: np.ndarray
    referenceDensity: float
    soundSpeed: float
    gravity: np.ndarray
    alpha: float = 0.01
    boundaryViscosityFactor: float = 0.0
    xsphEpsilon: float = 0.0
    densityFloor: float = 0.0         # kg/m^3
    densityDiffusion: str = 'none'
    diffusionDelta: float = 0.1
    wallExtrapolated: bool = False
    negativePressure: bool = False
    continuityCorrection: bool = False
    viscosityLimiter: bool = False
    cflNumber: float = 0.25
    maxTimeStep: float = 1.0
    densityFilterInterval: int = 0
    period: float = 0.0
    turbulenceClosure: str = 'none'   # 'deltaLes': the delta-LES-SPH closure
    particleShifting: bool = False    # Lind et al.'s shifting, its size CFL Ma (2h)^2 or 2 h |v| dt (local)
    shiftingMach: float = 0.1
    shiftingLocal: bool = False
    trackEnergy: bool = False         # the device steps keep the energy budget (src/pysurf/sphEnergy.py)
    compensatedSums: bool = False     # the momentum and continuity sums carry their rounding error
    kinematicViscosity: float = 1.0034e-6     # src/pysurf/constants.py:35, the closure's water term
    info: dict = field(default_factory=dict)

    @property
    def fluidCount(self) -> int:
        return int(np.count_nonzero(self.state.isFluid))


def latticePoints(lower, upper, spacing: float) -> np.ndarray:
    """Cell centres of a square lattice filling [lower, upper] (src/pysurf/sphParticles.py:289-312)."""
    axes = [np.arange(low + spacing / 2.0, high, spacing) for low, high in zip(lower, upper)]
    grids = np.meshgrid(*axes, indexing='xy')
    return np.column_stack([grid.ravel() for grid in grids])


def containerPositions(lower, upper, spacing: float, layers: int, openTop: bool) -> np.ndarray:
    """The wall shell of src/pysurf/sphBoundaries.py:96-124 (ContainerBoundary.positions)."""
    lower, upper = np.asarray(lower, dtype=float), np.asarray(upper, dtype=float)
    dim = len(lower)
    offsets = (np.arange(layers) + 0.5) * spacing
    axes = []
    for axis, (low, high) in enumerate(zip(lower, upper)):
        pieces = [low - offsets[::-1], np.arange(low + spacing / 2.0, high, spacing)]
        if not (openTop and axis == dim - 1):
            pieces.append(high + offsets)
        axes.append(np.concatenate(pieces))
    grids = np.meshgrid(*axes, indexing='xy')
    points = np.column_stack([grid.ravel() for grid in grids])
    interior = np.all((points > lower) & (points < upper), axis=1)
    if openTop:
        between = np.all((points[:, :-1] > lower[:-1]) & (points[:, :-1] < upper[:-1]), axis=1)
        interior = between & (points[:, -1] > lower[-1])
    return points[~interior]


def taitDensity(pressure, rho0: float, c0: float) -> np.ndarray:
    """src/pysurf/sphSolver.py:560-566."""
    stiffness = rho0 * c0 ** 2 / 7.0
    return rho0 * (1.0 + np.asarray(pressure) / stiffness) ** (1.0 / 7.0)


def hydrostaticDensity(depth, rho0: float, c0: float, g: float = GRAVITY) -> np.ndarray:
    """src/pysurf/sphSolver.py:1106-1120: the density carrying rho0 g z below the surface."""
    return taitDensity(rho0 * g * np.maximum(np.asarray(depth, dtype=float), 0.0), rho0, c0)


def damBreak(spacing: float = 0.02, seed: int = 0, kernelType: str = 'wendlandC2', diffusion: str = 'hydrostatic',
             smoothingRatio: float = 1.3) -> Case:
    """A 1.0 x 2.0 m water column in a 4.0 x 3.0 m tank, three layers of wall particles, the lattice
    jittered by U(-0.01, 0.01) spacings from a seed: 5,000 fluid particles at 0.02 m."""
    rng = np.random.default_rng(seed)
    fluid = latticePoints([0.0, 0.0], [1.0, 2.0], spacing)
    fluid = fluid + rng.uniform(-0.01 * spacing, 0.01 * spacing, size=fluid.shape)
    lower, upper = np.zeros(2), np.array([4.0, 3.0])
    wall = containerPositions(lower, upper, spacing, 3, True)
    rho0 = 1000.0
    height = 2.0
    c0 = 10.0 * math.sqrt(GRAVITY * height)
    state = ParticleState.assemble(fluid, wall, spacing, rho0)
    state.densities = hydrostaticDensity(height - state.positions[:, 1], rho0, c0)
    return Case('damBreak', state, ContainerBoundary(lower, upper, spacing, 3, True), 2, spacing,
                smoothingRatio * spacing, kernelType, lower, upper, rho0, c0, np.array([0.0, -GRAVITY]), alpha=0.01,
                densityDiffusion=diffusion, cflNumber=0.2, maxTimeStep=1.0,
                info={'tank': [4.0, 3.0], 'column': [1.0, 2.0], 'layers': 3})


def sloshingTank(tilt: float = 10.0, width: float = 0.2, height: float = 0.15, fill: float = 0.5,
                 spacing: float = 0.005, **scheme) -> Case:
    """The sloshing tank of the reference's GPU tests (tests/testSphGpu.py:441-457, built by
    src/pysurf/WaterSim/scenarios/sloshingTank.py:108-157): water below a surface tilted `tilt` degrees
    in a container with three wall layers, the default scheme (cubic spline at h = 1.3 dx, Shepard every
    30 steps, XSPH 0.5, alpha 0.1) with `scheme` overriding any Case field, and a step no longer than 1 ms."""
    slope = math.tan(math.radians(tilt))
    fillHeight = fill * height
    lower, upper = np.zeros(2), np.array([width, height])
    points = latticePoints(lower, upper, spacing)
    fluid = points[points[:, 1] < fillHeight + slope * (points[:, 0] - width / 2.0)]
    wall = containerPositions(lower, upper, spacing, 3, True)
    rho0 = FRESHWATER
    c0 = 10.0 * math.sqrt(GRAVITY * height)
    state = ParticleState.assemble(fluid, wall, spacing, rho0)
    surface = fillHeight + slope * (state.positions[:, 0] - width / 2.0)
    state.densities = hydrostaticDensity(surface - state.positions[:, 1], rho0, c0)
    ratio = scheme.pop('smoothingLengthRatio', 1.3)
    fields = dict(kernelType='cubicSpline', alpha=0.1, xsphEpsilon=0.5, cflNumber=0.25, maxTimeStep=1e-3,
                  densityFilterInterval=30)
    fields.update(scheme)
    kernelType = fields.pop('kernelType')
    if 'densityFloor' in fields:
        fields['densityFloor'] = fields['densityFloor'] * rho0    # given as a share of rho0
    return Case('sloshingTank', state, ContainerBoundary(lower, upper, spacing, 3, True), 2, spacing, ratio * spacing,
                kernelType, lower, upper, rho0, c0, np.array([0.0, -GRAVITY]), **fields,
                info={'tilt': tilt, 'fillHeight': fillHeight})


# -- the solitary wave over a plane beach -- #

def planeBeach(depth: float, toeX: float, slope: float, endX: float, startX: float = 0.0) -> Profile:
    """src/pysurf/bathymetry.py:115-140: flat to the toe, then a constant slope."""
    return Profile(np.array([startX, toeX, endX]), np.array([0.0, 0.0, (endX - toeX) * slope]), depth)


def profileSample(bed: Profile, spacing: float):
    """Points along the bed at equal arc length, both ends included (src/pysurf/bathymetry.py:272-293)."""
    lengths = np.hypot(np.diff(bed.x), np.diff(bed.z))
    arc = np.concatenate([[0.0], np.cumsum(lengths)])
    count = max(2, int(round(arc[-1] / spacing)) + 1)
    targets = np.linspace(0.0, arc[-1], count)
    return np.interp(targets, arc, bed.x), np.interp(targets, arc, bed.z)


def profileNormal(bed: Profile, x) -> np.ndarray:
    """The bed's upward unit normal (src/pysurf/bathymetry.py:233-250)."""
    slopes = np.diff(bed.z) / np.diff(bed.x)
    index = np.clip(np.searchsorted(bed.x, x, side='right') - 1, 0, slopes.size - 1)
    slope = slopes[index]
    length = np.sqrt(1.0 + slope ** 2)
    return np.stack([-slope / length, 1.0 / length], axis=-1)


def bedPositions(bed: Profile, spacing: float, layers: int, wallTop: float | None,
                 endWallTop: float | None) -> np.ndarray:
    """The 2D bed's layers and end walls (src/pysurf/sphBoundaries.py:196-215, BedBoundary._profilePositions)."""
    bedX, bedZ = profileSample(bed, spacing)
    normal = profileNormal(bed, bedX)
    blocks = [np.column_stack([bedX, bedZ]) - (layer + 0.5) * spacing * normal for layer in range(layers)]
    for wallX, top, side in ((bed.startX, wallTop, -1.0), (bed.endX, endWallTop, 1.0)):
        if top is None:
            continue
        bottom = float(bed.elevation(wallX)) - layers * spacing
        heights = np.arange(bottom + spacing / 2.0, top, spacing)
        for layer in range(layers):
            blocks.append(np.column_stack([np.full_like(heights, wallX + side * (layer + 0.5) * spacing), heights]))
    return np.vstack(blocks)


def solitaryWaveSpeed(height: float, depth: float) -> float:
    """c = sqrt(g (d + H)) (src/pysurf/waveTheory.py:192-196)."""
    return math.sqrt(GRAVITY * (depth + height))


def solitaryWaveDecay(height: float, depth: float) -> float:
    """kappa = sqrt(3 H / (4 d^3)) (src/pysurf/waveTheory.py:198-202)."""
    return math.sqrt(3.0 * height / (4.0 * depth ** 3))


def solitaryWaveProfile(x, height: float, depth: float, crestX: float) -> np.ndarray:
    """eta = H sech^2(kappa (x - x0)) (src/pysurf/waveTheory.py:204-225)."""
    argument = solitaryWaveDecay(height, depth) * (np.asarray(x, dtype=float) - crestX)
    return height / np.cosh(argument) ** 2


def solitaryWaveFluid(bed: Profile, height: float, crestX: float, spacing: float):
    """The lattice below the first-order solitary wave and its velocities (src/pysurf/waveMakers.py:258-329)."""
    depth = float(max(0.0, bed.stillWaterLevel - bed.elevation(crestX)))
    swl = bed.stillWaterLevel
    lower = [bed.startX, float(np.min(bed.z))]
    upper = [bed.endX, swl + height + spacing]
    points = latticePoints(lower, upper, spacing)
    bedZ = bed.elevation(points[:, 0])
    surface = swl + solitaryWaveProfile(points[:, 0], height, depth, crestX)
    keep = (points[:, 1] >= bedZ + (0.5 - 1e-9) * spacing) & (points[:, 1] < surface)
    positions = points[keep]
    x, y = positions[:, 0], positions[:, 1]
    celerity = solitaryWaveSpeed(height, depth)
    kappa = solitaryWaveDecay(height, depth)
    eta = solitaryWaveProfile(x, height, depth, crestX)
    etaSlope = -2.0 * kappa * eta * np.tanh(kappa * (x - crestX))
    u = celerity * eta / (depth + eta)
    w = -(y - bed.elevation(x)) * celerity * depth * etaSlope / (depth + eta) ** 2
    return positions, np.column_stack([u, w])


def solitaryBeach(particlesPerDepth: int = 64, depth: float = 1.0, height: float = 0.45, crestX: float = 10.0,
                  toeX: float = 15.0, slope: float = 1.0 / 15.0, length: float = 60.0, smoothingRatio: float = 3.0,
                  layers: int | None = None) -> Case:
    """A first-order (Boussinesq sech^2) solitary wave of H/d = 0.45 at x0 = 10 d over a 1:15 beach from
    x = 15 d, 60 d long, run with the deltaSph scheme of src/pysurf/BreakingWave.py:722-725: Wendland C2 at
    h = 3 dx, hydrostatic diffusion, the continuity correction, extrapolated walls, the viscosity limiter and a
    density floor of 0.9 rho0, alpha = 0.01, c0 = 10 c.  Layers default to the facade's max(3, ceil(2h/dx))."""
    s = depth / particlesPerDepth
    layers = max(3, math.ceil(2.0 * smoothingRatio - 1e-9)) if layers is None else layers
    bed = planeBeach(depth, toeX, slope, length)
    wallTop = depth + 3.0 * height
    boundary = BedBoundary(bed, s, nLayers=layers, wallTop=wallTop, endWallTop=None, wallX=bed.startX)
    fluid, velocities = solitaryWaveFluid(bed, height, crestX, s)
    rho0 = FRESHWATER
    state = ParticleState.assemble(fluid, bedPositions(bed, s, layers, wallTop, None), s, rho0, velocities)
    c0 = 10.0 * solitaryWaveSpeed(height, depth)
    surface = depth + solitaryWaveProfile(state.positions[:, 0], height, depth, crestX)
    state.densities = hydrostaticDensity(surface - state.positions[:, 1], rho0, c0)
    margin = (layers + 1.0) * s
    return Case('solitaryBeach', state, boundary, 2, s, smoothingRatio * s, 'wendlandC2',
                np.array([-margin, -margin]), np.array([length + margin, wallTop]), rho0, c0,
                np.array([0.0, -GRAVITY]), alpha=0.01, densityFloor=0.9 * rho0, densityDiffusion='hydrostatic',
                wallExtrapolated=True, continuityCorrection=True, viscosityLimiter=True, cflNumber=0.25,
                maxTimeStep=1.0,
                info={'depth': depth, 'H/d': height / depth, 'crestX': crestX, 'toeX': toeX, 'slope': slope,
                      'length': length, 'ppd': particlesPerDepth, 'layers': layers})


def extrudedBeach(particlesPerDepth: int = 8, width: float = 1.75, depth: float = 1.0, height: float = 0.6,
                  crestX: float = 2.5, toeX: float = 4.0, slope: float = 1.0 / 15.0, length: float = 20.0,
                  smoothingRatio: float = 3.0) -> Case:
    """The beach of `solitaryBeach` in 3D: its 2D start (first-order solitary wave, bed layers, offshore
    wall) repeated across a periodic y axis `width` long, one lattice column a spacing, the bed a
    BedBoundary over the profile with no side walls (src/pysurf/sphBoundaries.py:295-344, periodic), the
    deltaSph scheme at h = 3 dx.  The period must exceed twice the support (4 h)."""
    flat = solitaryBeach(particlesPerDepth, depth, height, crestX, toeX, slope, length, smoothingRatio)
    s = flat.spacing
    columns = int(round(width / s))
    if columns * s <= 4.0 * flat.smoothingLength:
        raise ValueError('the periodic width must exceed twice the kernel support (4 h)')
    width = columns * s
    ys = (np.arange(columns) + 0.5) * s

    def extrude(points):
        n = len(points)
        out = np.empty((n * columns, 3))
        out[:, 0] = np.tile(points[:, 0], columns)
        out[:, 1] = np.repeat(ys, n)
        out[:, 2] = np.tile(points[:, 1], columns)
        return out

    st, nf = flat.state, flat.fluidCount
    fluid, walls = extrude(st.positions[:nf]), extrude(st.positions[nf:])
    velocities = np.zeros((len(fluid), 3))
    velocities[:, 0] = np.tile(st.velocities[:nf, 0], columns)
    velocities[:, 2] = np.tile(st.velocities[:nf, 1], columns)
    state = ParticleState.assemble(fluid, walls, s, flat.referenceDensity, velocities)
    state.densities = np.concatenate([np.tile(st.densities[:nf], columns), np.tile(st.densities[nf:], columns)])
    bed = flat.boundary
    boundary = BedBoundary(bed.bathymetry, s, nLayers=bed.nLayers, wallTop=bed.wallTop, width=width,
                           endWallTop=None, periodic=True, wallX=bed.wallX)
    lower, upper = flat.domainMin, flat.domainMax
    info = dict(flat.info, width=width, columns=columns)
    return Case('extrudedBeach', state, boundary, 3, s, flat.smoothingLength, flat.kernelType,
                np.array([lower[0], 0.0, lower[1]]), np.array([upper[0], width, upper[1]]), flat.referenceDensity,
                flat.soundSpeed, np.array([0.0, 0.0, -GRAVITY]), alpha=flat.alpha, densityFloor=flat.densityFloor,
                densityDiffusion=flat.densityDiffusion, wallExtrapolated=True, continuityCorrection=True,
                viscosityLimiter=True, cflNumber=flat.cflNumber, maxTimeStep=flat.maxTimeStep, period=width,
                info=info)


def gaussianRidge(depth: float = 1.0, ridgeHeight: float = 0.6, ridgeWidth: float = 3.0, angle: float = 25.0,
                  length: float = 40.0, width: float = 10.0, ridgeX: float = 20.0):
    """The bed z_b(x, y) = ridgeHeight d exp(-xi^2 / (2 sigma^2)) of a Gaussian ridge whose axis crosses
    (ridgeX, width / 2) at `angle` degrees to the y axis (the crest line of a wave travelling along +x),
    xi the distance from the axis (the bed of HeightField.fromFunction, src/pysurf/bathymetry.py:480-517).
    Returns (elevation(x, y), gradient(x, y) -> (dz/dx, dz/dy))."""
    a = math.radians(angle)
    ca, sa = math.cos(a), math.sin(a)
    peak, sigma2 = ridgeHeight * depth, (ridgeWidth * depth) ** 2

    def distance(x, y):
        return (np.asarray(x, dtype=float) - ridgeX) * ca - (np.asarray(y, dtype=float) - 0.5 * width) * sa

    def elevation(x, y):
        xi = distance(x, y)
        return peak * np.exp(-xi * xi / (2.0 * sigma2))

    def gradient(x, y):
        xi = distance(x, y)
        dz = -elevation(x, y) * xi / sigma2
        return dz * ca, -dz * sa

    return elevation, gradient


def heightTable(elevation, bounds, gridSpacing: float, stillWaterLevel: float, padding: int = 2) -> HeightTable:
    """A height field sampled on a grid `padding` cells past its bounds, as the device's cubic
    convolution reads it (src/pysurf/bathymetry.py:480-517)."""
    startX, endX, startY, endY = bounds
    x = startX + gridSpacing * np.arange(-padding, int(math.ceil((endX - startX) / gridSpacing)) + padding + 1)
    y = startY + gridSpacing * np.arange(-padding, int(math.ceil((endY - startY) / gridSpacing)) + padding + 1)
    gx, gy = np.meshgrid(x, y, indexing='xy')
    return HeightTable(x, y, elevation(gx, gy), tuple(bounds), stillWaterLevel)


def heightFieldPositions(elevation, gradient, bounds, spacing: float, layers: int, wallTop: float,
                         floor: float) -> np.ndarray:
    """Boundary particles of a height-field tank (src/pysurf/sphBoundaries.py:498-595): the bed's layers
    on the lattice's columns, each offset along the local normal by (layer + 1/2) s, then walls on all
    four sides whose columns stand behind their planes at (layer + 1/2) s, on the fluid lattice's
    heights from below the bed's deepest layer to `wallTop`; the side walls run past the end walls."""
    startX, endX, startY, endY = bounds
    xs = np.arange(startX + 0.5 * spacing, endX, spacing)
    ys = np.arange(startY + 0.5 * spacing, endY, spacing)
    gx, gy = (g.ravel() for g in np.meshgrid(xs, ys, indexing='xy'))
    zx, zy = gradient(gx, gy)
    norm = np.sqrt(1.0 + zx * zx + zy * zy)
    normal = np.column_stack([-zx / norm, -zy / norm, 1.0 / norm])
    surface = np.column_stack([gx, gy, elevation(gx, gy)])
    blocks = [surface - (layer + 0.5) * spacing * normal for layer in range(layers)]
    heights = np.arange(floor - (layers + 1) * spacing + 0.5 * spacing, wallTop, spacing)

    def wall(lineX, lineY):
        bottom = elevation(np.clip(lineX, startX, endX), np.clip(lineY, startY, endY)) - layers * spacing
        x, y = np.repeat(lineX, heights.size), np.repeat(lineY, heights.size)
        z = np.tile(heights, lineX.size)
        keep = z > np.repeat(bottom, heights.size)
        return np.column_stack([x[keep], y[keep], z[keep]])

    offsets = (np.arange(layers) + 0.5) * spacing
    for offset in offsets:
        blocks.append(wall(np.full(ys.size, startX - offset), ys))
        blocks.append(wall(np.full(ys.size, endX + offset), ys))
    along = np.concatenate([startX - offsets[::-1], xs, endX + offsets])
    for offset in offsets:
        blocks.append(wall(along, np.full(along.size, startY - offset)))
        blocks.append(wall(along, np.full(along.size, endY + offset)))
    return np.vstack(blocks)


def ridgeWave3D(particlesPerDepth: int = 32, depth: float = 1.0, height: float = 0.5, crestX: float = 8.0,
                ridgeHeight: float = 0.6, ridgeWidth: float = 3.0, angle: float = 25.0, length: float = 40.0,
                width: float = 10.0, ridgeX: float = 20.0, smoothingRatio: float = 3.0,
                layers: int | None = None) -> Case:
    """A first-order solitary wave of H/d = 0.5 crossing a Gaussian ridge (0.6 d high, sigma = 3 d, its axis
    at 25 degrees to the crest) in a 40 d x 10 d tank with walls on all sides, 32 particles per depth, run
    with the deltaSph scheme of src/pysurf/BreakingWave3D.py:656-662 (Wendland C2 at h = 3 dx, hydrostatic
    diffusion, the continuity correction, extrapolated walls, the viscosity limiter, density floor 0.9 rho0).
    The fluid fills the lattice's cells from the bed to the wave's surface (the layout of
    src/pysurf/BreakingWave3D.py:630-700 without start packing); crest-zone splitting is a separate step."""
    s = depth / particlesPerDepth
    layers = max(3, math.ceil(2.0 * smoothingRatio - 1e-9)) if layers is None else layers
    bounds = (0.0, length, 0.0, width)
    elevation, gradient = gaussianRidge(depth, ridgeHeight, ridgeWidth, angle, length, width, ridgeX)
    floor = 0.0
    wallTop = depth + 3.0 * height
    table = heightTable(elevation, bounds, 0.5 * s, depth)
    boundary = HeightFieldBoundary(table, s, nLayers=layers, wallTop=wallTop)
    # fluid: lattice cells from the bed to the surface d + eta(x)
    xs = np.arange(0.5 * s, length, s)
    ys = np.arange(0.5 * s, width, s)
    zs = np.arange(floor + 0.5 * s, depth + height + s, s)
    gx, gy, gz = (g.ravel() for g in np.meshgrid(xs, ys, zs, indexing='ij'))
    bedZ = elevation(gx, gy)
    surface = depth + solitaryWaveProfile(gx, height, depth, crestX)
    keep = (gz >= bedZ + (0.5 - 1e-9) * s) & (gz < surface)
    fluid = np.column_stack([gx[keep], gy[keep], gz[keep]])
    x, z, bed = fluid[:, 0], fluid[:, 2], bedZ[keep]
    celerity = solitaryWaveSpeed(height, depth)
    kappa = solitaryWaveDecay(height, depth)
    eta = solitaryWaveProfile(x, height, depth, crestX)
    etaSlope = -2.0 * kappa * eta * np.tanh(kappa * (x - crestX))
    u = celerity * eta / (depth + eta)
    w = -(z - bed) * celerity * depth * etaSlope / (depth + eta) ** 2
    velocities = np.column_stack([u, np.zeros_like(u), w])
    rho0 = FRESHWATER
    walls = heightFieldPositions(elevation, gradient, bounds, s, layers, wallTop, floor)
    state = ParticleState.assemble(fluid, walls, s, rho0, velocities)
    c0 = 10.0 * celerity
    top = depth + solitaryWaveProfile(state.positions[:, 0], height, depth, crestX)
    state.densities = hydrostaticDensity(top - state.positions[:, 2], rho0, c0)
    margin = (layers + 2.0) * s
    return Case('ridgeWave3D', state, boundary, 3, s, smoothingRatio * s, 'wendlandC2',
                np.array([-margin, -margin, floor - margin]), np.array([length + margin, width + margin, wallTop]),
                rho0, c0, np.array([0.0, 0.0, -GRAVITY]), alpha=0.01, densityFloor=0.9 * rho0,
                densityDiffusion='hydrostatic', wallExtrapolated=True, continuityCorrection=True,
                viscosityLimiter=True, cflNumber=0.25, maxTimeStep=1.0,
                info={'depth': depth, 'H/d': height / depth, 'crestX': crestX, 'ridge': [ridgeHeight, ridgeWidth, angle],
                      'ridgeX': ridgeX, 'tank': [length, width], 'ppd': particlesPerDepth, 'layers': layers})


def ridgeSection(case: Case, y: float) -> Profile:
    """The ridge's bed along x at fixed y, through the height table's x positions inside the tank
    and its two ends (HeightField.section, src/pysurf/bathymetry.py:719-731): the bed profile a
    section's breaking tracker reads."""
    info, table = case.info, case.boundary.field
    ridgeHeight, ridgeWidth, angle = info['ridge']
    length, width = info['tank']
    elevation, _ = gaussianRidge(float(info['depth']), ridgeHeight, ridgeWidth, angle, length, width,
                                 float(info['ridgeX']))
    startX, endX = float(table.bounds[0]), float(table.bounds[1])
    inside = table.x[(table.x > startX + 1e-9) & (table.x < endX - 1e-9)]
    x = np.concatenate([[startX], inside, [endX]])
    return Profile(x, elevation(x, np.full_like(x, float(y))), table.stillWaterLevel)


def refineCrestZone(sums, case: Case, share: float = 0.3, lengthRatio: float = 0.5) -> int:
    """The crest-zone split of the 3D ridge workload: every fluid particle not yet split, in a
    column (one spacing across) whose surface stands more than `share` H above still water, splits
    into 2^dim daughters of h times `lengthRatio` (src/pysurf/sphRefinement.py:136-190), on the
    device.  Returns how many split."""
    info, s = case.info, case.spacing
    depth = float(info['depth'])
    height = float(info['H/d']) * depth
    lower, upper = case.domainMin, case.domainMax
    nx = int(math.ceil((upper[0] - lower[0]) / s))
    ny = int(math.ceil((upper[1] - lower[1]) / s)) if case.dimensions == 3 else 1
    fluidMass = float(np.max(case.state.masses[case.state.isFluid]))
    return sums.splitCrestZone(lower[0], lower[1], s, nx, ny, depth + share * height, 0.999 * fluidMass,
                               case.referenceDensity, lengthRatio)


def pairSumsFor(case: Case, cellsPerSupport: int | None = None, device: int = 0):
    """A PairSums set up for a case: the switches WcsphSolver.__init__ sets (src/pysurf/sphSolver.py:1499-1518)
    and the physics WcsphSolver.advance sets (src/pysurf/sphSolver.py:1970-1972)."""
    from pysurf_b200.sphGpu import PairSums
    sums = PairSums(case.dimensions, case.smoothingLength, case.domainMin, case.domainMax, case.period,
                    device=device, kernelType=case.kernelType)
    if cellsPerSupport is not None:
        sums.setCellsPerSupport(cellsPerSupport)
    sums.setDiffusion(case.densityDiffusion, case.diffusionDelta, case.soundSpeed, case.referenceDensity,
                      abs(float(case.gravity[-1])))
    sums.setWallPressure(case.wallExtrapolated)
    sums.setNegativePressure(case.negativePressure)
    sums.setContinuityCorrection(case.continuityCorrection)
    sums.setViscosityLimiter(case.viscosityLimiter)
    sums.setClosure(case.turbulenceClosure == 'deltaLes', case.soundSpeed, case.referenceDensity,
                    case.kinematicViscosity)
    sums.setShifting(case.particleShifting, case.shiftingMach, case.spacing, case.soundSpeed, case.shiftingLocal)
    sums.setEnergyBudget(case.trackEnergy)
    if case.compensatedSums:
        sums.setCompensatedSums(True)
    sums.setPhysics(case.referenceDensity, case.soundSpeed, case.alpha, case.boundaryViscosityFactor, case.gravity,
                    case.xsphEpsilon, case.densityFloor)
    return sums
