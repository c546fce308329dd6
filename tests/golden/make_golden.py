"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run in a container that holds the reference checkout (``python tests/golden/make_golden.py
/path/to/reference``).  It imports the reference's own float64 array formulation
(src/pysurf/sphSolver.py), its numba neighbour list (src/pysurf/sphCompiled.py), its boundaries
(src/pysurf/sphBoundaries.py), its refinement (src/pysurf/sphRefinement.py) and its scenario
builders, runs them on the inputs its own tests use (tests/testSphGpu.py:32-63 and the sloshing
tank of tests/testSphGpu.py:441-457), and saves inputs and outputs as compressed .npz files.

The reference's package __init__ pulls plotting and unit libraries that the sums do not need, so
the package object, ``pysurf.constants`` (g = 9.80665, src/pysurf/constants.py:29-38) and
``pysurf.figures`` are stubbed; every module used below is the reference's, unmodified.

Nothing at test time imports the reference: the tests read these files only.
"""
from __future__ import annotations

import math
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def loadReference(root: str):
    package = types.ModuleType('pysurf')
    package.__path__ = [os.path.join(root, 'src', 'pysurf')]
    sys.modules['pysurf'] = package
    constants = types.ModuleType('pysurf.constants')
    constants.gravity = 9.80665
    constants.freshwaterDensity = 998.2
    constants.freshwaterKinematicViscosity = 1.0034e-6
    constants.seawaterDensity = 1025.0
    sys.modules['pysurf.constants'] = constants
    package.constants = constants
    figures = types.ModuleType('pysurf.figures')
    sys.modules['pysurf.figures'] = figures
    package.figures = figures


rho0, c0, alpha, epsilon = 1000.0, 20.0, 0.1, 0.5


def cloud(dimensions, periodic, seed=3, kernelType='cubicSpline'):
    """The random cloud of tests/testSphGpu.py:32-63 (offset 25 m from the origin)."""
    from pysurf.sphKernels import createKernel
    from pysurf.sphNeighbors import neighborPairs
    from pysurf.sphSolver import taitEquationOfState
    rng = np.random.default_rng(seed)
    count, spacing = (600, 0.04) if dimensions == 2 else (900, 0.045)
    extent = np.full(dimensions, spacing * count ** (1.0 / dimensions))
    positions = 25.0 + rng.uniform(0.0, 1.0, size=(count, dimensions)) * extent
    period = None
    if periodic:
        positions[:, 1] -= 25.0
        period = float(extent[1])
    h = (2.0 if kernelType == 'wendlandC2' else 1.3) * spacing
    velocities = rng.normal(0.0, 1.0, size=(count, dimensions))
    densities = rho0 * (1.0 + rng.uniform(-0.01, 0.01, size=count))
    masses = rho0 * spacing ** dimensions * (1.0 + rng.uniform(-0.05, 0.05, size=count))
    isFluid = rng.uniform(size=count) < 0.8
    pressures = taitEquationOfState(densities, rho0, c0)
    i, j = neighborPairs(positions, 2.0 * h, period)
    separation = positions[i] - positions[j]
    if period is not None:
        separation[:, 1] -= period * np.round(separation[:, 1] / period)
    distance = np.linalg.norm(separation, axis=1)
    kernel = createKernel(kernelType, dimensions)
    return dict(kernelType=kernelType, positions=positions, period=period, h=h, velocities=velocities,
                densities=densities, masses=masses, isFluid=isFluid, pressures=pressures, i=i, j=j,
                separation=separation, distance=distance, values=kernel.evaluateBatch(distance, h),
                gradients=kernel.gradientBatch(separation, distance, h), kernel=kernel)


def strainedFlow(case):
    """tests/testSphGpu.py:199-206: a linear flow under noise."""
    positions = case['positions']
    dimensions = positions.shape[1]
    return (positions - positions.mean(axis=0)) @ np.random.default_rng(11).normal(
        size=(dimensions, dimensions)).T + 0.3 * case['velocities']


def makeClouds():
    from pysurf import sphCompiled
    from pysurf.sphSolver import (artificialViscosity, continuityRate, correctionMatrices, densityDiffusionRate,
                                  extrapolatedWallPressure, limitedVelocityDifference, pairAccelerations,
                                  renormalizedDensityGradient, shepardDensity, taitDensity, velocityGradients,
                                  xsphVelocity)
    out = {}
    for dimensions, periodic in [(2, False), (3, False), (3, True)]:
        for kernelType in ('cubicSpline', 'wendlandC2'):
            tag = f'{dimensions}d_{"p" if periodic else "o"}_{kernelType}'
            case = cloud(dimensions, periodic, kernelType=kernelType)
            i, j, fluid = case['i'], case['j'], case['isFluid']
            n = len(fluid)
            gravity = np.zeros(dimensions)
            gravity[-1] = -9.81
            factor = 0.3
            rec = dict(positions=case['positions'], velocities=case['velocities'], densities=case['densities'],
                       masses=case['masses'], isFluid=fluid, pressures=case['pressures'], h=case['h'],
                       period=case['period'] or 0.0, kernel=1 if kernelType == 'wendlandC2' else 0)
            # Plain accelerations (tests/testSphGpu.py:79-99)
            viscosity = artificialViscosity(case['velocities'][i] - case['velocities'][j], case['separation'],
                                            case['distance'], 0.5 * (case['densities'][i] + case['densities'][j]),
                                            case['h'], c0, alpha)
            viscosity[~(fluid[i] & fluid[j])] *= factor
            acc = pairAccelerations(case['masses'], case['densities'], case['pressures'], i, j, case['gradients'],
                                    viscosity, n)
            acc[fluid] += gravity
            acc[~fluid] = 0.0
            rec['accelerations'] = acc
            # Limited accelerations and velocity gradients (tests/testSphGpu.py:101-133)
            strained = strainedFlow(case)
            G = velocityGradients(case['masses'], case['densities'], strained, i, j, case['separation'],
                                  case['gradients'], fluid)
            relative = strained[i] - strained[j]
            rec_ = limitedVelocityDifference(relative, case['separation'], case['distance'], case['h'], G[i], G[j])
            boundaryPairs = ~(fluid[i] & fluid[j])
            rec_[boundaryPairs] = relative[boundaryPairs]
            viscosity = artificialViscosity(relative, case['separation'], case['distance'],
                                            0.5 * (case['densities'][i] + case['densities'][j]), case['h'], c0,
                                            alpha, rec_)
            viscosity[boundaryPairs] *= factor
            accL = pairAccelerations(case['masses'], case['densities'], case['pressures'], i, j, case['gradients'],
                                     viscosity, n)
            accL[fluid] += gravity
            accL[~fluid] = 0.0
            rec['strained'] = strained
            rec['velocityGradients'] = G
            rec['limitedAccelerations'] = accL
            # Continuity, plain and corrected (tests/testSphGpu.py:135-168)
            rec['continuity'] = continuityRate(case['masses'], case['velocities'], i, j, case['gradients'], n,
                                               fluid[i] | fluid[j])
            L = correctionMatrices(case['masses'], case['densities'], i, j, case['separation'], case['gradients'],
                                   fluid)
            rec['corrections'] = L
            rec['correctedContinuity'] = continuityRate(case['masses'], case['velocities'], i, j, case['gradients'],
                                                        n, fluid[i] | fluid[j], L)
            # Diffusive continuity (tests/testSphGpu.py:170-187)
            plain = rec['continuity']
            for mode in ('molteni', 'hydrostatic'):
                gravityMagnitude = 9.81 if mode == 'hydrostatic' else None
                rec[f'diffusive_{mode}'] = plain + densityDiffusionRate(
                    case['masses'], case['densities'], i, j, case['separation'], case['distance'],
                    case['gradients'], n, case['h'], c0, 0.1, rho0, gravityMagnitude, fluid[i] & fluid[j])
            # Antuono (tests/testSphGpu.py:189-208)
            gradients = renormalizedDensityGradient(case['masses'], case['densities'], i, j, case['gradients'], L,
                                                    fluid)
            rec['densityGradients'] = gradients
            rec['diffusive_antuono'] = plain + densityDiffusionRate(
                case['masses'], case['densities'], i, j, case['separation'], case['distance'], case['gradients'], n,
                case['h'], c0, 0.1, rho0, None, fluid[i] & fluid[j], gradients)
            # Wall pressure (tests/testSphGpu.py:306-318) and the boundary's density from it
            wall = extrapolatedWallPressure(case['densities'], case['pressures'], i, j, case['separation'],
                                            case['values'], fluid, gravity)
            rec['wallPressure'] = wall
            rec['wallDensity'] = np.where(fluid, case['densities'], taitDensity(wall, rho0, c0))
            # XSPH and Shepard (tests/testSphGpu.py:368-388)
            pairs = fluid[i] & fluid[j]
            rec['xsph'] = xsphVelocity(case['velocities'], case['masses'], case['densities'], i[pairs], j[pairs],
                                       case['values'][pairs], epsilon)
            rec['shepard'] = shepardDensity(case['masses'], case['densities'], i, j, case['values'],
                                            case['kernel'].evaluate(0.0, case['h']))
            # The reference's compiled neighbour rows at the support (src/pysurf/sphCompiled.py:133-234)
            offsets, neighbors = sphCompiled.neighborList(case['positions'], 2.0 * case['h'], case['period'] or 0.0)
            rec['offsets'] = np.asarray(offsets, dtype=np.int64)
            rec['neighbors'] = np.asarray(neighbors, dtype=np.int32)
            # The cKDTree pair set (src/pysurf/sphNeighbors.py:28-78)
            rec['pairCount'] = np.array(len(i))
            for key, value in rec.items():
                out[f'{tag}/{key}'] = np.asarray(value)
    np.savez_compressed(os.path.join(HERE, 'clouds.npz'), **out)


def makeCellKeys():
    from pysurf.sphSolver import cellOrderKey
    positions = np.array([[0.5, 0.5, 0.5], [1.5, 0.5, 0.5], [0.5, 1.5, 0.5], [0.5, 0.5, 1.5], [4.5, 0.5, 0.5],
                          [-0.5, 0.5, 0.5]])
    rng = np.random.default_rng(5)
    random3 = rng.uniform(-3.0, 40.0, size=(2000, 3))
    random2 = rng.uniform(-3.0, 60.0, size=(2000, 2))
    np.savez_compressed(os.path.join(HERE, 'cellkeys.npz'),
                        known3=positions, keys3=cellOrderKey(positions, 1.0, (4, 3, 2)),
                        known2=positions[:3, :2], keys2=cellOrderKey(positions[:3, :2], 1.0, (4, 3, 1)),
                        random3=random3, randomKeys3=cellOrderKey(random3, 0.37, (57, 23, 9)),
                        random2=random2, randomKeys2=cellOrderKey(random2, 0.09375, (700, 40, 1)))


def makeEnforcement():
    """tests/testSphGpu.py:645-712: host enforcement of a reef bed (2D, 3D) and a ridge height field."""
    from pysurf.bathymetry import Bathymetry, HeightField
    from pysurf.sphBoundaries import BedBoundary, HeightFieldBoundary
    from pysurf.sphParticles import ParticleSystem
    out = {}
    for dimensions in (2, 3):
        rng = np.random.default_rng(7)
        bed = Bathymetry.reefBreak(depth=1.0, toeX=2.0, faceSlope=0.2, reefDepth=0.3, reefLength=2.0)
        s, width = 0.05, (0.6 if dimensions == 3 else None)
        boundary = BedBoundary(bed, s, nLayers=3, wallTop=1.5, width=width,
                               endWallTop=1.5 if dimensions == 2 else None)
        count = 4000
        fluid = np.column_stack([rng.uniform(bed.startX - 0.2, bed.endX + 0.2, count)]
                                + ([rng.uniform(-0.1, 0.7, count)] if dimensions == 3 else [])
                                + [rng.uniform(-1.2, 1.2, count)])
        host = ParticleSystem.assemble(fluid, boundary.positions(), s, 1000.0, rng.normal(0.0, 1.0, (count, dimensions)))
        boundary.attachPiston(host)
        boundary.movePiston(host, bed.startX + 0.03, 0.4)
        tag = f'bed{dimensions}d'
        keep = host.isFluid.copy()
        out[f'{tag}/positions'] = host.positions[keep].copy()
        out[f'{tag}/velocities'] = host.velocities[keep].copy()
        out[f'{tag}/bedX'] = bed.x.copy()
        out[f'{tag}/bedZ'] = bed.z.copy()
        clearance = 0.25 * boundary.spacing
        sideWalls = boundary.width is not None and not boundary.periodic
        endLimit = bed.endX - clearance if boundary.endWallTop is not None else bed.endX
        mask = boundary._pistonMask
        pistonSpeed = float(host.velocities[mask, 0][0])
        out[f'{tag}/params'] = np.array([clearance, float(sideWalls), float(boundary.width or 0.0),
                                         float(boundary.wallTop is not None), float(boundary.wallX), pistonSpeed,
                                         float(endLimit)])
        boundary.enforce(host)
        out[f'{tag}/enforcedPositions'] = host.positions[keep].copy()
        out[f'{tag}/enforcedVelocities'] = host.velocities[keep].copy()
    rng = np.random.default_rng(11)
    field = HeightField.ridge(0.5, endX=8.0, halfWidth=2.0, gridSpacing=1.0 / 16.0)
    s = 0.125
    boundary = HeightFieldBoundary(field, s, nLayers=3, wallTop=1.5)
    count = 6000
    fluid = np.column_stack([rng.uniform(-0.2, 8.2, count), rng.uniform(-0.2, 2.2, count), rng.uniform(-0.1, 1.2, count)])
    host = ParticleSystem.assemble(fluid, boundary.positions(), s, 1000.0, rng.normal(0.0, 1.0, (count, 3)))
    keep = host.isFluid.copy()
    out['field/positions'] = host.positions[keep].copy()
    out['field/velocities'] = host.velocities[keep].copy()
    out['field/table'] = field.z.copy()
    clearance = 0.25 * s
    startX, endX, startY, endY = field.bounds
    out['field/params'] = np.array([float(field.x[0]), float(field.y[0]), field.spacingX, field.spacingY, clearance,
                                    startY + clearance, endY - clearance, float(boundary.offshoreWall),
                                    startX + clearance, endX - clearance if boundary.endWall else endX])
    boundary.enforce(host)
    out['field/enforcedPositions'] = host.positions[keep].copy()
    out['field/enforcedVelocities'] = host.velocities[keep].copy()
    np.savez_compressed(os.path.join(HERE, 'enforce.npz'), **out)


def sloshing(backend='numpy', tilt=10.0, **options):
    """tests/testSphGpu.py:441-457: a 0.2 x 0.15 m tank half full at 5 mm spacing."""
    from pysurf.sphSolver import WcsphSolver
    from pysurf.WaterSim.scenarios.sloshingTank import SloshingTankConfig, createSloshingTank
    tank = SloshingTankConfig(tankWidth=0.2, tankHeight=0.15, fillRatio=0.5, initialTiltDeg=tilt,
                              particleSpacing=0.005)
    config, particles, boundary = createSloshingTank(tank)
    config.backend = backend
    config.maxTimeStep = 1e-3
    for name, value in options.items():
        setattr(config, name, value)
    solver = WcsphSolver(config, boundary=boundary)
    solver.initialize(particles)
    return solver, particles, boundary


deltaContinuity = dict(densityFilterInterval=0, xsphEpsilon=0.0, wallPressure='extrapolated',
                       continuityCorrection=True, densityFloor=0.9)


def recordRun(out, tag, solver, particles, steps, boundaryRecord):
    config = solver.config
    out[f'{tag}/positions'] = particles.positions.copy()
    out[f'{tag}/velocities'] = particles.velocities.copy()
    out[f'{tag}/densities'] = particles.densities.copy()
    out[f'{tag}/masses'] = particles.masses.copy()
    out[f'{tag}/isFluid'] = particles.isFluid.copy()
    modes = {'none': 0, 'molteni': 1, 'hydrostatic': 2, 'antuono': 3}
    out[f'{tag}/config'] = np.array([
        config.dimensions, 1.0 if config.kernelType == 'wendlandC2' else 0.0, config.smoothingLength,
        config.referenceDensity, solver.speedOfSound, config.alphaViscosity, config.boundaryViscosityFactor,
        config.xsphEpsilon, config.densityFloor * config.referenceDensity, modes[config.densityDiffusion],
        config.diffusionDelta, float(config.wallPressure == 'extrapolated'), float(config.negativePressure),
        float(config.continuityCorrection), float(config.viscosityLimiter), config.cflNumber, config.maxTimeStep,
        float(config.densityFilterInterval), float(config.periodicWidth or 0.0)])
    out[f'{tag}/gravity'] = np.asarray(config.gravity, dtype=float)
    out[f'{tag}/domain'] = np.array([list(config.domainMin), list(config.domainMax)], dtype=float)
    for key, value in boundaryRecord.items():
        out[f'{tag}/boundary_{key}'] = np.asarray(value)
    dts = []
    for _ in range(steps):
        state = solver.step()
        dts.append(state.dt)
    out[f'{tag}/steps'] = np.array(steps)
    out[f'{tag}/dts'] = np.array(dts)
    out[f'{tag}/finalPositions'] = particles.positions.copy()
    out[f'{tag}/finalVelocities'] = particles.velocities.copy()
    out[f'{tag}/finalDensities'] = particles.densities.copy()
    out[f'{tag}/finalPressures'] = particles.pressures.copy()
    out[f'{tag}/finalAccelerations'] = particles.accelerations.copy()


def containerRecord(boundary):
    return dict(kind=1, lower=boundary.containerMin, upper=boundary.containerMax, openTop=int(boundary.openTop))


def makeRuns():
    """Host steps of the reference's float64 numpy solver, the runs its GPU tests compare against."""
    out = {}
    runs = {
        'plain': dict(),                                                  # Shepard filter and XSPH
        'limited': dict(viscosityLimiter=True),
        'deltaHydrostatic': dict(densityDiffusion='hydrostatic', **deltaContinuity),
        'deltaAntuono': dict(deltaContinuity, continuityCorrection=False, densityDiffusion='antuono'),
        'tension': dict(negativePressure=True),
        'deltaWendland': dict(kernelType='wendlandC2', smoothingLengthRatio=2.0, densityDiffusion='hydrostatic',
                              viscosityLimiter=True, **deltaContinuity),
    }
    for tag, options in runs.items():
        solver, particles, boundary = sloshing(**options)
        if tag == 'tension':
            particles.densities[particles.isFluid] *= 0.998
        steps = 30 if tag != 'plain' else 40
        recordRun(out, tag, solver, particles, steps, containerRecord(boundary))
    # A solitary wave over a flat channel bed, the deltaSph scheme at h = 3 dx (tests/testSphGpu.py:714-750)
    from pysurf import constants, waveTheory
    from pysurf.bathymetry import Bathymetry
    from pysurf.sphBoundaries import BedBoundary
    from pysurf.sphParticles import ParticleSystem
    from pysurf.sphSolver import SimulationConfig, WcsphSolver
    from pysurf.waveMakers import solitaryWaveFluid
    depth, height, spacing = 1.0, 0.3, 1.0 / 8.0
    crestX = waveTheory.solitaryWaveHalfLength(height, depth, 0.01)
    channel = Bathymetry([0.0, 12.0], [0.0, 0.0], stillWaterLevel=depth)
    boundary = BedBoundary(channel, spacing, nLayers=6, wallTop=1.9, endWallTop=1.9)
    fluid, velocities = solitaryWaveFluid(channel, height, crestX, spacing)
    particles = ParticleSystem.assemble(fluid, boundary.positions(), spacing, constants.freshwaterDensity, velocities)
    config = SimulationConfig(domainMin=np.array([-0.5, -0.5]), domainMax=np.array([12.5, 1.9]),
                              particleSpacing=spacing, maxTimeStep=1.0, smoothingLengthRatio=3.0,
                              kernelType='wendlandC2', densityDiffusion='hydrostatic', viscosityLimiter=True,
                              speedOfSound=10.0 * waveTheory.solitaryWaveSpeed(height, depth), alphaViscosity=0.01,
                              backend='numpy', initialSurface=lambda x: depth + waveTheory.solitaryWaveProfile(
                                  x, height, depth, crestX), **deltaContinuity)
    solver = WcsphSolver(config, boundary=boundary)
    solver.initialize(particles)
    clearance = 0.25 * spacing
    bedRecord = dict(kind=2, bedX=channel.x, bedZ=channel.z,
                     params=[clearance, 0.0, 0.0, 1.0, float(boundary.wallX), 0.0, channel.endX - clearance])
    recordRun(out, 'bedDelta', solver, particles, 40, bedRecord)
    np.savez_compressed(os.path.join(HERE, 'runs.npz'), **out)


def ridgeWave(particlesPerDepth=6):
    """A small 3D tank for BreakingWave3D's deltaSph scheme on the host: a solitary wave of H/d = 0.4
    approaching a Gaussian ridge (0.3 d high, sigma 0.8 d, its axis at 25 degrees to the crest) over a
    height-field bed, 5 d x 1.5 d, built by the reference's own facade (src/pysurf/BreakingWave3D.py:630-700)
    without start packing, its solver on the numpy backend."""
    from pysurf.bathymetry import HeightField
    from pysurf.BreakingWave3D import BreakingWave3D
    angle = math.radians(25.0)

    def ridge(x, y):
        across = (x - 3.0) * math.cos(angle) + (y - 0.75) * math.sin(angle)
        return 0.3 * np.exp(-across ** 2 / (2.0 * 0.8 ** 2))

    field = HeightField.fromFunction(ridge, (0.0, 5.0, 0.0, 1.5), 1.0 / 32.0, stillWaterLevel=1.0)
    wave = BreakingWave3D(field, 0.4, 2.0, particlesPerDepth=particlesPerDepth, backend='numpy', startPacking=False,
                          endTime=0.1)
    wave.build()
    return wave


def heightFieldRecord(boundary):
    field, clearance = boundary.field, 0.25 * boundary.spacing
    startX, endX, startY, endY = field.bounds
    return dict(kind=3, table=field.z, gridX=field.x, gridY=field.y, bounds=list(field.bounds),
                stillWaterLevel=field.stillWaterLevel, spacing=boundary.spacing, layers=boundary.nLayers,
                wallTop=boundary.wallTop, offshoreWall=int(bool(boundary.offshoreWall)),
                endWall=int(bool(boundary.endWall)),
                params=[float(field.x[0]), float(field.y[0]), float(field.x[1] - field.x[0]),
                        float(field.y[1] - field.y[0]), clearance, startY + clearance, endY - clearance,
                        float(bool(boundary.offshoreWall)), startX + clearance,
                        endX - clearance if boundary.endWall else endX])


def makeRuns3D():
    """Host steps of the reference's float64 numpy solver in 3D: the ridge tank above under the deltaSph
    scheme, as it starts and after its crest splits into daughters of h / 2 (WcsphSolver.refine,
    src/pysurf/sphSolver.py:1994-2040), the runs tests/testBreakingWave3D.py:298-347 take on the GPU."""
    out = {}
    for tag, steps, split in (('ridge', 25, False), ('ridgeSplit', 15, True)):
        wave = ridgeWave()
        solver, particles = wave.solver, wave.particles
        if split:
            # the crest zone: fluid within a half length of the crest and above the still water level
            x = particles.positions
            zone = particles.isFluid & (np.abs(x[:, 0] - wave.crestX) < 0.5) & (x[:, 2] > 1.0)
            out[f'{tag}/splitCount'] = np.array(solver.refine(zone, lengthRatio=0.5))
        out[f'{tag}/lengths'] = np.array(particles.lengths if particles.lengths is not None
                                         else np.full(particles.nParticles, solver.config.smoothingLength))
        recordRun(out, tag, solver, particles, steps, heightFieldRecord(wave.boundary))
        print(tag, particles.nParticles, 'particles', int(particles.isFluid.sum()), 'fluid', steps, 'steps')
    np.savez_compressed(os.path.join(HERE, 'runs3d.npz'), **out)


def makeSplit():
    """src/pysurf/sphRefinement.py:136-190 on a small 2D and 3D set, h kept and h halved."""
    from pysurf.sphParticles import ParticleSystem
    from pysurf.sphRefinement import splitParticles
    out = {}
    for dimensions in (2, 3):
        for ratio in (1.0, 0.5):
            rng = np.random.default_rng(21 + dimensions)
            s = 0.05
            fluid = 3.0 + rng.uniform(0.0, 1.0, (300, dimensions))
            wall = rng.uniform(0.0, 1.0, (60, dimensions))
            particles = ParticleSystem.assemble(fluid, wall, s, 1000.0, rng.normal(0.0, 1.0, (300, dimensions)))
            particles.densities = 1000.0 + rng.uniform(-5, 5, len(particles.densities))
            particles.pressures = rng.uniform(0, 10, len(particles.densities))
            mask = rng.uniform(size=len(particles.densities)) < 0.3
            tag = f'split{dimensions}d_{ratio}'
            for name in ('positions', 'velocities', 'accelerations', 'densities', 'pressures', 'masses', 'isFluid'):
                out[f'{tag}/{name}'] = getattr(particles, name).copy()
            out[f'{tag}/mask'] = mask
            count = splitParticles(particles, mask, 1000.0, 1.3 * s, ratio)
            out[f'{tag}/count'] = np.array(count)
            for name in ('positions', 'velocities', 'accelerations', 'densities', 'pressures', 'masses', 'isFluid',
                         'lengths'):
                out[f'{tag}/split_{name}'] = getattr(particles, name).copy()
    np.savez_compressed(os.path.join(HERE, 'split.npz'), **out)


def makeBeach():
    """The solitary-wave-on-a-plane-beach start at 8 particles per depth, as the reference builds it."""
    from pysurf import constants, waveTheory
    from pysurf.bathymetry import Bathymetry
    from pysurf.sphBoundaries import BedBoundary, ContainerBoundary
    from pysurf.sphParticles import ParticleSystem, latticePoints
    from pysurf.sphSolver import hydrostaticDensity
    from pysurf.waveMakers import solitaryWaveFluid
    out = {}
    depth, height, ppd = 1.0, 0.45, 8
    s = depth / ppd
    beach = Bathymetry.planeBeach(depth=depth, toeX=15.0, slope=1.0 / 15.0, endX=60.0)
    layers = 6
    boundary = BedBoundary(beach, s, nLayers=layers, wallTop=depth + 3.0 * height, endWallTop=None)
    fluid, velocities = solitaryWaveFluid(beach, height, 10.0, s)
    particles = ParticleSystem.assemble(fluid, boundary.positions(), s, constants.freshwaterDensity, velocities)
    c0 = 10.0 * waveTheory.solitaryWaveSpeed(height, depth)
    surface = depth + waveTheory.solitaryWaveProfile(particles.positions[:, 0], height, depth, 10.0)
    densities = hydrostaticDensity(surface - particles.positions[:, -1], constants.freshwaterDensity, c0)
    out['beach/positions'] = particles.positions
    out['beach/velocities'] = particles.velocities
    out['beach/isFluid'] = particles.isFluid
    out['beach/masses'] = particles.masses
    out['beach/densities'] = densities
    # The dam break's tank: a 1 x 2 m column in a 4 x 3 m container, 3 layers, at 0.1 m
    tank = ContainerBoundary(np.zeros(2), np.array([4.0, 3.0]), 0.1, nLayers=3, openTop=True)
    out['dam/boundary'] = tank.positions()
    out['dam/column'] = latticePoints([0.0, 0.0], [1.0, 2.0], 0.1)
    np.savez_compressed(os.path.join(HERE, 'beach.npz'), **out)


def breakingShapes(bed, s, seed=5):
    """Fluid position sets that exercise the breaking measures: a still beach, a steep crest, a lip
    leaning one and three spacings over the face, and the same jittered."""
    rng = np.random.default_rng(seed)
    swl = bed.stillWaterLevel
    x = np.arange(0.5 * s, 40.0, s)
    z = np.arange(0.5 * s, 2.0, s)
    gx, gz = np.meshgrid(x, z, indexing='xy')
    gx, gz = gx.ravel(), gz.ravel()
    bedZ = np.interp(gx, bed.x, bed.z)
    shapes = {}
    for name, crest, height, lip in (('still', 20.0, 0.0, 0), ('steep', 22.0, 0.45, 0), ('lip1', 24.0, 0.5, 1),
                                     ('lip3', 25.0, 0.55, 3)):
        surface = swl + height * np.exp(-((gx - crest) / 1.2) ** 2 * np.where(gx > crest, 6.0, 1.0))
        keep = (gz >= bedZ + 0.5 * s) & (gz < surface)
        points = np.column_stack([gx[keep], gz[keep]])
        if lip:
            # a tongue of water leaning `lip` spacings ahead of the face near the crest's top
            top = swl + height
            tongue = [(crest + 0.4 + (k + 1) * s, top - (j + 0.5) * s) for k in range(lip + 3) for j in range(3)]
            points = np.vstack([points, np.asarray(tongue)])
        shapes[name] = points
        shapes[name + '_jitter'] = points + rng.uniform(-0.2 * s, 0.2 * s, points.shape)
    return shapes


def makeBreaking():
    """The breaking measures of src/pysurf/waveBreaking.py ('cells' face) on synthetic fluid shapes over a
    1:15 beach, and a tracker fed a sequence of them."""
    from pysurf.bathymetry import Bathymetry
    from pysurf.waveBreaking import (BreakingTracker, freeSurfaceProfile, frontFaceLean, troughAhead,
                                     waterlineX)
    out = {}
    s = 1.0 / 16.0
    beach = Bathymetry.planeBeach(depth=1.0, toeX=15.0, slope=1.0 / 15.0, endX=60.0)
    out['bed/x'], out['bed/z'] = np.asarray(beach.x), np.asarray(beach.z)
    shapes = breakingShapes(beach, s)
    for name, points in shapes.items():
        centers, elevation = freeSurfaceProfile(points, beach.startX, beach.endX, s)
        crest = int(np.nanargmax(elevation))
        crestX = float(centers[crest])
        out[f'{name}/positions'] = points
        out[f'{name}/centers'] = centers
        out[f'{name}/elevation'] = elevation
        out[f'{name}/lean'] = np.array(frontFaceLean(points, crestX, beach.stillWaterLevel, s, 1.0))
        out[f'{name}/trough'] = np.array(troughAhead(centers, elevation, crestX, 2.0))
        out[f'{name}/waterline'] = np.array(waterlineX(points, beach, 2.0 * s))
    tracker = BreakingTracker(beach, s, faceReach=1.0, searchFromX=15.0)
    sequence = ['still', 'steep', 'lip1', 'steep', 'lip1', 'lip1_jitter', 'lip1', 'lip3', 'steep']
    for k, name in enumerate(sequence):
        tracker.update(0.1 * (k + 1), shapes[name])
    out['sequence'] = np.array(sequence)
    point = tracker.breakingPoint
    out['tracker/crestX'] = np.asarray(tracker.crestX)
    out['tracker/crestHeight'] = np.asarray(tracker.crestHeight)
    out['tracker/lean'] = np.asarray(tracker.lean)
    out['tracker/waterline'] = np.asarray(tracker.waterline)
    out['tracker/maxRunup'] = np.array(tracker.maxRunup)
    out['tracker/point'] = np.array([point.time, point.lean, point.crestX, point.crestHeight, point.depth,
                                     point.troughHeight]) if point is not None else np.full(6, np.nan)
    np.savez_compressed(os.path.join(HERE, 'breaking.npz'), **out)


def makeClosure():
    """The delta-LES-SPH closure (src/pysurf/sphSolver.py:1232-1326 and its use in _computeRates, 1615-1745):
    coefficients, accelerations and continuity on the six clouds under a strained flow, and a
    sloshing run with turbulenceClosure 'deltaLes'."""
    from pysurf import constants
    from pysurf.sphSolver import (artificialViscosity, closureCoefficients, closureViscosity, continuityRate,
                                  densityDiffusionRate, harmonicMean, pairAccelerations, velocityGradients)
    out = {}
    nu = constants.freshwaterKinematicViscosity
    for dimensions, periodic in [(2, False), (3, False), (3, True)]:
        for kernelType in ('cubicSpline', 'wendlandC2'):
            tag = f'{dimensions}d_{"p" if periodic else "o"}_{kernelType}'
            case = cloud(dimensions, periodic, kernelType=kernelType)
            i, j, fluid = case['i'], case['j'], case['isFluid']
            n = len(fluid)
            gravity = np.zeros(dimensions)
            gravity[-1] = -9.81
            factor = 0.3
            strained = strainedFlow(case)
            G = velocityGradients(case['masses'], case['densities'], strained, i, j, case['separation'],
                                  case['gradients'], fluid)
            alphas, deltas = closureCoefficients(G, fluid, case['h'], c0)
            relative = strained[i] - strained[j]
            viscosity = artificialViscosity(relative, case['separation'], case['distance'],
                                            0.5 * (case['densities'][i] + case['densities'][j]), case['h'], c0, alpha)
            boundaryPairs = ~(fluid[i] & fluid[j])
            viscosity[boundaryPairs] *= factor
            fp = ~boundaryPairs
            fi, fj = i[fp], j[fp]
            viscosity[fp] += closureViscosity(relative[fp], case['separation'][fp], case['distance'][fp],
                                              case['densities'][fi], case['densities'][fj], case['h'], c0, rho0,
                                              alphas[fi], alphas[fj], nu)
            acc = pairAccelerations(case['masses'], case['densities'], case['pressures'], i, j, case['gradients'],
                                    viscosity, n)
            acc[fluid] += gravity
            acc[~fluid] = 0.0
            rate = continuityRate(case['masses'], strained, i, j, case['gradients'], n, fluid[i] | fluid[j])
            rate = rate + densityDiffusionRate(case['masses'], case['densities'], i, j, case['separation'],
                                               case['distance'], case['gradients'], n, case['h'], c0,
                                               harmonicMean(deltas[i], deltas[j]), rho0, 9.81, fluid[i] & fluid[j])
            for key, value in dict(alphas=alphas, deltas=deltas, accelerations=acc, continuity=rate).items():
                out[f'{tag}/{key}'] = np.asarray(value)
    out['viscosity'] = np.array(nu)
    runs = {}
    solver, particles, boundary = sloshing(turbulenceClosure='deltaLes', densityDiffusion='hydrostatic',
                                           **deltaContinuity)
    recordRun(runs, 'closure', solver, particles, 30, containerRecord(boundary))
    out.update(runs)
    np.savez_compressed(os.path.join(HERE, 'closure.npz'), **out)


def latticeCloud(dimensions, kernelType, seed=11):
    """Water on a jittered square lattice over three layers of wall particles, its top a free
    surface: a shift acts inside it and the free-surface rules at its top."""
    from pysurf.sphKernels import createKernel
    from pysurf.sphNeighbors import neighborPairs
    from pysurf.sphSolver import taitEquationOfState
    rng = np.random.default_rng(seed)
    spacing = 0.02
    shape = (24, 18) if dimensions == 2 else (10, 8, 9)
    axes = [np.arange(k) * spacing for k in shape]
    grids = np.meshgrid(*axes, indexing='ij')
    lattice = np.column_stack([g.ravel() for g in grids]) + 5.0
    positions = lattice + rng.uniform(-0.15 * spacing, 0.15 * spacing, lattice.shape)
    isFluid = lattice[:, -1] >= 5.0 + 3 * spacing - 1e-9
    positions[~isFluid] = lattice[~isFluid]
    count = len(positions)
    h = (2.0 if kernelType == 'wendlandC2' else 1.3) * spacing
    velocities = rng.normal(0.0, 0.1, size=(count, dimensions))
    velocities[~isFluid] = 0.0
    densities = rho0 * (1.0 + rng.uniform(-0.005, 0.005, size=count))
    masses = np.full(count, rho0 * spacing ** dimensions)
    i, j = neighborPairs(positions, 2.0 * h, None)
    separation = positions[i] - positions[j]
    distance = np.linalg.norm(separation, axis=1)
    kernel = createKernel(kernelType, dimensions)
    return dict(positions=positions, velocities=velocities, densities=densities, masses=masses, isFluid=isFluid,
                pressures=taitEquationOfState(densities, rho0, c0), h=h, spacing=spacing, i=i, j=j,
                separation=separation, distance=distance, values=kernel.evaluateBatch(distance, h),
                gradients=kernel.gradientBatch(separation, distance, h), kernel=kernel)


def makeShifting():
    """Particle shifting (src/pysurf/sphSolver.py:824-1010, and its step in _integrate, 1760-1785): the
    fields, the displacement, the density and velocity changes on the six clouds, and a sloshing run
    with particleShifting on."""
    from pysurf.sphSolver import shiftedVelocityChange, shiftingDisplacement, shiftingFields
    out = {}
    for dimensions in (2, 3):
        for kernelType in ('cubicSpline', 'wendlandC2'):
            tag = f'{dimensions}d_{kernelType}'
            case = latticeCloud(dimensions, kernelType)
            for key in ('positions', 'velocities', 'densities', 'masses', 'isFluid', 'pressures', 'h'):
                out[f'{tag}/{key}'] = np.asarray(case[key])
            out[f'{tag}/kernel'] = np.array(1 if kernelType == 'wendlandC2' else 0)
            i, j, fluid = case['i'], case['j'], case['isFluid']
            n = len(fluid)
            spacing = case['spacing']
            spacingKernel = float(case['kernel'].evaluate(spacing, case['h']))
            fields = shiftingFields(case['masses'], case['densities'], i, j, case['separation'], case['values'],
                                    case['gradients'], n, spacingKernel)
            size = 0.2 * 0.1 * (2.0 * case['h']) ** 2
            shift, densityChange = shiftingDisplacement(*fields, i, j, case['values'], fluid, size, case['h'],
                                                        kernelType)
            velocityChange = shiftedVelocityChange(case['masses'], case['densities'], case['velocities'], i, j,
                                                   case['gradients'], shift, fluid[i] & fluid[j])
            names = ('gradient', 'plain', 'divergence', 'densityGradient')
            for key, value in list(zip(names, fields)) + [('shift', shift), ('densityChange', densityChange),
                                                          ('velocityChange', velocityChange)]:
                out[f'{tag}/{key}'] = np.asarray(value)
            out[f'{tag}/spacingKernel'] = np.array(spacingKernel)
            out[f'{tag}/size'] = np.array(size)
    runs = {}
    solver, particles, boundary = sloshing(particleShifting=True, densityDiffusion='hydrostatic', **deltaContinuity)
    runs['shifting/mach'] = np.array(solver.config.shiftingMach)
    runs['shifting/spacing'] = np.array(solver.config.particleSpacing)
    recordRun(runs, 'shifting', solver, particles, 30, containerRecord(boundary))
    out.update(runs)
    np.savez_compressed(os.path.join(HERE, 'shifting.npz'), **out)


def solitaryChannel(**options):
    """tests/testSphEnergy.py:27-52: a solitary wave of H/d = 0.3 in a 12 m channel at 8 particles per
    depth on the deltaSph scheme, its options replaced by `options`; returns the solver, the particles
    and the bed's record."""
    from pysurf import constants, waveTheory
    from pysurf.bathymetry import Bathymetry
    from pysurf.sphBoundaries import BedBoundary
    from pysurf.sphParticles import ParticleSystem
    from pysurf.sphSolver import SimulationConfig, WcsphSolver
    from pysurf.waveMakers import solitaryWaveFluid
    depth, height, spacing = 1.0, 0.3, 1.0 / 8.0
    crestX = waveTheory.solitaryWaveHalfLength(height, depth, 0.01)
    channel = Bathymetry([0.0, 12.0], [0.0, 0.0], stillWaterLevel=depth)
    boundary = BedBoundary(channel, spacing, nLayers=6, wallTop=1.9, endWallTop=1.9)
    fluid, velocities = solitaryWaveFluid(channel, height, crestX, spacing)
    particles = ParticleSystem.assemble(fluid, boundary.positions(), spacing, constants.freshwaterDensity, velocities)
    scheme = dict(kernelType='wendlandC2', smoothingLengthRatio=3.0, densityFilterInterval=0,
                  densityDiffusion='hydrostatic', xsphEpsilon=0.0, wallPressure='extrapolated',
                  continuityCorrection=True, densityFloor=0.9, viscosityLimiter=True, alphaViscosity=0.01)
    scheme.update(options)
    config = SimulationConfig(domainMin=np.array([-1.0, -1.0]), domainMax=np.array([13.0, 1.9]),
                              particleSpacing=spacing, maxTimeStep=1.0, backend='numpy',
                              speedOfSound=10.0 * waveTheory.solitaryWaveSpeed(height, depth),
                              initialSurface=lambda x: depth + waveTheory.solitaryWaveProfile(x, height, depth, crestX),
                              **scheme)
    solver = WcsphSolver(config, boundary=boundary)
    solver.initialize(particles)
    clearance = 0.25 * spacing
    record = dict(kind=2, bedX=channel.x, bedZ=channel.z,
                  params=[clearance, 0.0, 0.0, 1.0, float(boundary.wallX), 0.0, channel.endX - clearance])
    return solver, particles, record


def makeEnergy():
    """The energy budget (src/pysurf/sphEnergy.py; its terms in src/pysurf/sphSolver.py:1650-1852 and
    1909-1936): the elastic energy and its slope on a table of densities, and the array solver's
    budget over runs that reach every term the device keeps."""
    from pysurf.sphEnergy import elasticEnergy, elasticSlope, energyTerms
    out = {'terms': np.array(energyTerms)}
    densities = np.array([985.0, 999.0, 999.999, 1000.0, 1000.0 + 1e-8, 1000.2, 1003.0, 1030.0, 1100.0])
    out['elastic/densities'] = densities
    for tension in (False, True):
        out[f'elastic/energy_{int(tension)}'] = elasticEnergy(densities, rho0, c0, tension)
    before = np.array([1001.0, 1002.0, 1002.0, 999.0, 990.0, 1000.0])
    after = np.array([1003.0, 1002.0 + 1e-9, 1002.0, 998.0, 1010.0, 1000.0 + 1e-5])
    out['elastic/before'], out['elastic/after'] = before, after
    for tension in (False, True):
        out[f'elastic/slope_{int(tension)}'] = elasticSlope(before, after, rho0, c0, tension)
    out['elastic/rho0'], out['elastic/c0'] = np.array(rho0), np.array(c0)
    closureForms = {'published': dict(densityDiffusion='antuono', turbulenceClosure='deltaLes', alphaViscosity=0.0,
                                      viscosityLimiter=False),
                    'hybrid': dict(densityDiffusion='antuono', turbulenceClosure='deltaLes')}

    def tracked(tag, solver, particles, steps, record):
        solver.trackEnergy()
        state = solver.currentState
        out[f'{tag}/startEnergy'] = np.array([state.kineticEnergy, state.potentialEnergy, solver.elasticEnergy])
        recordRun(out, tag, solver, particles, steps, record)
        state = solver.currentState
        out[f'{tag}/endEnergy'] = np.array([state.kineticEnergy, state.potentialEnergy, solver.elasticEnergy])
        budget = solver.energyBudget
        out[f'{tag}/budget'] = np.array([budget[name] for name in energyTerms])
        out[f'{tag}/closure'] = np.array(int(solver.config.turbulenceClosure == 'deltaLes'))
        out[f'{tag}/shifting'] = np.array([int(solver.config.particleShifting), solver.config.shiftingMach,
                                           solver.config.particleSpacing])

    for tag, options in [('channel', {}), ('uncorrected', dict(continuityCorrection=False)),
                         ('published', closureForms['published']), ('hybrid', closureForms['hybrid'])]:
        solver, particles, record = solitaryChannel(**options)
        tracked(tag, solver, particles, 20 if tag == 'uncorrected' else 40, record)
    # the Shepard filter, XSPH and viscosity against the walls; then shifting
    solver, particles, boundary = sloshing(boundaryViscosityFactor=0.5)
    tracked('filtered', solver, particles, 40, containerRecord(boundary))
    solver, particles, boundary = sloshing(particleShifting=True, densityDiffusion='hydrostatic', **deltaContinuity)
    tracked('shifted', solver, particles, 30, containerRecord(boundary))
    # the container's clamp (a corner of the fluid thrown at the walls) and the density floor under
    # tension (the surface's top row below it)
    solver, particles, boundary = sloshing(negativePressure=True, densityDiffusion='hydrostatic', **deltaContinuity)
    fluid = particles.isFluid
    corner = fluid & (particles.positions[:, 0] < 0.012) & (particles.positions[:, 1] < 0.012)
    particles.positions[corner] -= 0.003
    particles.velocities[corner] = [-0.8, -0.8]
    top = fluid & (particles.positions[:, 1] > particles.positions[fluid, 1].max() - 0.003)
    particles.densities[top] = 0.88 * particles.densities[top]
    tracked('clamped', solver, particles, 30, containerRecord(boundary))
    np.savez_compressed(os.path.join(HERE, 'energy.npz'), **out)


def makeFrames():
    """A run's frame files (src/pysurf/sphFrames.py:38-121), written by the reference's FrameWriter
    from the split fixture's particles, with a field and a scalar; and its checkpoint layout
    (src/pysurf/BreakingWave3D.py:204, 785-858): the format tag and the ParticleSystem fields."""
    import dataclasses
    import json
    import tempfile
    from pysurf import BreakingWave3D
    from pysurf.sphFrames import FrameWriter, readFrame
    from pysurf.sphParticles import ParticleSystem
    out = {}
    split = np.load(os.path.join(HERE, 'split.npz'))
    for dimensions in (2, 3):
        tag, key = f'frames{dimensions}d', f'split{dimensions}d_0.5'
        p = ParticleSystem(**{name: split[f'{key}/split_{name}'] for name in
                              ('positions', 'velocities', 'accelerations', 'densities', 'pressures', 'masses',
                               'isFluid', 'lengths')})
        fluidCount = int(p.isFluid.sum())
        with tempfile.TemporaryDirectory() as directory:
            writer = FrameWriter(directory)
            writer.write(0.25, p, step=7, fields={'ids': np.arange(fluidCount)}, scalars={'energy': 1.5})
            writer.write(0.5, p, step=9)
            for frame in (0, 1):
                for name, values in readFrame(directory, frame).items():
                    out[f'{tag}/frame{frame}_{name}'] = values
            with open(os.path.join(directory, 'frames.json'), encoding='utf-8') as handle:
                out[f'{tag}/index'] = np.array(handle.read())
        for name in ('positions', 'velocities', 'masses', 'isFluid', 'lengths'):
            out[f'{tag}/state_{name}'] = getattr(p, name)
    out['checkpoint/format'] = np.array(BreakingWave3D.checkpointFormat)
    out['checkpoint/particleFields'] = np.array([f.name for f in dataclasses.fields(ParticleSystem)])
    np.savez_compressed(os.path.join(HERE, 'frames.npz'), **out)


def makeMerge():
    """mergeParticles (src/pysurf/sphRefinement.py:192-311): a lattice with its boundary, split in part
    (h kept, and h halved), jittered, then merged in part; a second level split and merged; and a
    merge straight after a split."""
    from pysurf.sphParticles import ParticleSystem
    from pysurf.sphRefinement import mergeParticles, splitParticles
    out = {}
    fields = ('positions', 'velocities', 'accelerations', 'densities', 'pressures', 'masses', 'isFluid', 'lengths')
    for dimensions in (2, 3):
        for ratio, twice in ((1.0, False), (0.5, False), (0.5, True)):
            rng = np.random.default_rng(40 + dimensions + (2 if twice else 0) + int(ratio * 4))
            s = 0.05
            side = 12 if dimensions == 2 else 6
            axes = [np.arange(side) * s + 0.5 * s for _ in range(dimensions)]
            fluid = np.stack(np.meshgrid(*axes, indexing='ij'), axis=-1).reshape(-1, dimensions) + 0.3
            wall = rng.uniform(0.0, 0.25, (40, dimensions))
            particles = ParticleSystem.assemble(fluid, wall, s, 1000.0, rng.normal(0.0, 1.0, (len(fluid), dimensions)))
            n = len(particles.masses)
            particles.densities = 1000.0 + rng.uniform(-5, 5, n)
            particles.pressures = rng.uniform(0, 10, n)
            particles.accelerations = rng.normal(0.0, 1.0, (n, dimensions))
            referenceMass = 1000.0 * s ** dimensions
            length = 1.3 * s
            splitParticles(particles, rng.uniform(size=n) < 0.7, 1000.0, length, ratio)
            if twice:
                splitParticles(particles, rng.uniform(size=len(particles.masses)) < 0.5, 1000.0, length, ratio)
            count = len(particles.masses)
            fluidRows = particles.isFluid
            particles.positions[fluidRows] += rng.uniform(-0.1, 0.1, (int(fluidRows.sum()), dimensions)) * s
            particles.velocities[fluidRows] += rng.normal(0.0, 0.2, (int(fluidRows.sum()), dimensions))
            particles.densities = 1000.0 + rng.uniform(-5, 5, count)
            mask = rng.uniform(size=count) < 0.85
            tag = f'merge{dimensions}d_{ratio}{"_twice" if twice else ""}'
            for name in fields:
                out[f'{tag}/{name}'] = np.array(getattr(particles, name))
            out[f'{tag}/mask'] = mask
            out[f'{tag}/reference'] = np.array([1000.0, referenceMass, length, ratio])
            result = mergeParticles(particles, mask, 1000.0, referenceMass, length, ratio)
            out[f'{tag}/groups'] = np.array(result.groups)
            out[f'{tag}/removedEnergy'] = np.array(result.removedEnergy)
            out[f'{tag}/source'] = np.asarray(result.source)
            for name in fields:
                out[f'{tag}/merged_{name}'] = np.array(getattr(particles, name))
    np.savez_compressed(os.path.join(HERE, 'merge.npz'), **out)


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('PYSURF_REFERENCE', '')
    if not root or not os.path.isdir(root):
        raise SystemExit('Give the reference checkout: make_golden.py /path/to/reference [fixture ...]')
    loadReference(root)
    makers = {'cellkeys': makeCellKeys, 'clouds': makeClouds, 'enforce': makeEnforcement, 'split': makeSplit,
              'beach': makeBeach, 'runs': makeRuns, 'breaking': makeBreaking, 'closure': makeClosure,
              'shifting': makeShifting, 'energy': makeEnergy, 'frames': makeFrames,
              'merge': makeMerge, 'runs3d': makeRuns3D}
    for name in (sys.argv[2:] or list(makers)):
        makers[name]()
    for name in sorted(os.listdir(HERE)):
        if name.endswith('.npz'):
            print(name, os.path.getsize(os.path.join(HERE, name)))


if __name__ == '__main__':
    main()
