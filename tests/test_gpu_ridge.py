"""The 3D target workload on the device, run against the reference's own float64 host steps and the
float64 oracle.

* The reference's BreakingWave3D facade builds a small ridge tank (a solitary wave approaching a
  Gaussian ridge over a height-field bed, deltaSph scheme, walls six layers deep) and its numpy solver
  steps it, as it starts and after its crest splits into daughters of h / 2 (tests/golden/runs3d.npz,
  made by tests/golden/make_golden.py).  The device steps the same inputs.
* The benchmark's own ridge (cases.ridgeWave3D: the 25-degree Gaussian ridge, walled tank, deltaSph
  scheme) in a shortened tank at 6 particles per depth, stepped by the device and by the oracle, whole
  and after the device's crest-zone split.

Tolerances are those the reference holds its float32 device to against the numpy solver
(tests/testSphGpu.py:503-517, 578-590): positions 1e-6 m, velocities and densities 1e-3, time 1e-4.
"""
import math

import numpy as np
import pytest

from conftest import golden, goldenTags
from oracle import oracle
from pysurf_b200 import cases
from pysurf_b200.state import HeightFieldBoundary, HeightTable, ParticleState

pytestmark = pytest.mark.gpu

RUNS = goldenTags('runs3d.npz')
MODES = ['none', 'molteni', 'hydrostatic', 'antuono']


def caseFromRun(r) -> cases.Case:
    (dim, kind, h, rho0, c0, alpha, bf, xsph, floor, mode, delta, wall, tension, corrected, limited, cfl, maxdt,
     interval, period) = r['config']
    n = len(r['masses'])
    state = ParticleState(r['positions'].copy(), r['velocities'].copy(), np.zeros_like(r['positions']),
                          r['densities'].copy(), np.zeros(n), r['masses'].copy(), r['isFluid'].copy())
    state.lengths = r['lengths'].copy()
    table = HeightTable(r['boundary_gridX'], r['boundary_gridY'], r['boundary_table'], tuple(r['boundary_bounds']),
                        float(r['boundary_stillWaterLevel']))
    boundary = HeightFieldBoundary(table, float(r['boundary_spacing']), int(r['boundary_layers']),
                                   float(r['boundary_wallTop']), bool(r['boundary_offshoreWall']),
                                   bool(r['boundary_endWall']))
    domain = r['domain']
    return cases.Case('ridgeRun', state, boundary, int(dim), float(r['boundary_spacing']), h,
                      'wendlandC2' if int(kind) == 1 else 'cubicSpline', domain[0], domain[1], rho0, c0, r['gravity'],
                      alpha=alpha, boundaryViscosityFactor=bf, xsphEpsilon=xsph, densityFloor=floor,
                      densityDiffusion=MODES[int(mode)], diffusionDelta=delta, wallExtrapolated=bool(wall),
                      negativePressure=bool(tension), continuityCorrection=bool(corrected),
                      viscosityLimiter=bool(limited), cflNumber=cfl, maxTimeStep=maxdt,
                      densityFilterInterval=int(interval), period=period)


def fieldParams(boundary: HeightFieldBoundary):
    """The oracle's height-field enforcement for a boundary, as PairSums.setBoundary hands it to the device."""
    field, clearance = boundary.field, 0.25 * boundary.spacing
    startX, endX, startY, endY = field.bounds
    return ('field', oracle.fieldParams(field.z, float(field.x[0]), float(field.y[0]), field.spacingX, field.spacingY,
                                        clearance, startY + clearance, endY - clearance, bool(boundary.offshoreWall),
                                        startX + clearance, endX - clearance if boundary.endWall else endX))


def stepperFor(case):
    return oracle.Stepper(case.dimensions, case.kernelType, case.smoothingLength, case.referenceDensity,
                          case.soundSpeed, case.alpha, case.gravity, case.boundaryViscosityFactor, case.xsphEpsilon,
                          case.densityFloor, case.densityDiffusion, case.diffusionDelta, case.wallExtrapolated,
                          case.negativePressure, case.continuityCorrection, case.viscosityLimiter, case.cflNumber,
                          case.maxTimeStep, 0.0, case.densityFilterInterval, fieldParams(case.boundary))


def assertFollows(out, time, ref, refTime):
    assert time == pytest.approx(refTime, rel=1e-4)
    assert np.abs(out['positions'] - ref['positions']).max() < 1e-6
    assert np.abs(out['velocities'] - ref['velocities']).max() < 1e-3
    assert np.abs(out['densities'] - ref['densities']).max() < 1e-3


@pytest.mark.parametrize('tag', RUNS)
def test_ridge_runs_follow_the_reference_host_steps(tag):
    r = golden('runs3d.npz', tag)
    case = caseFromRun(r)
    steps = int(r['steps'])
    sums = cases.pairSumsFor(case)
    state = case.state.copy()
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    time, step, _ = sums.advance(0.0, 0, math.inf, steps, float(state.lengths.min()), case.cflNumber,
                                 case.maxTimeStep)
    assert step == steps
    out = sums.pullState()
    if tag == 'ridgeSplit':
        assert out['lengths'].min() == 0.5 * case.smoothingLength
        assert out['masses'].sum() == r['masses'].sum()
    ref = {'positions': r['finalPositions'], 'velocities': r['finalVelocities'], 'densities': r['finalDensities']}
    assertFollows(out, time, ref, float(np.sum(r['dts'])))


def shortRidge():
    # the benchmark's ridge and scheme in a 12 d x 3 d tank, the crest 3 d ahead of the ridge's axis
    return cases.ridgeWave3D(6, length=12.0, width=3.0, crestX=4.0, ridgeX=7.0)


def test_the_ridge_workload_follows_the_oracle():
    case = shortRidge()
    steps = 30
    sums = cases.pairSumsFor(case)
    state = case.state.copy()
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    time, step, _ = sums.advance(0.0, 0, math.inf, steps, case.smoothingLength, case.cflNumber, case.maxTimeStep)
    assert step == steps
    out = sums.pullState()
    ref = {k: np.array(getattr(case.state, k), copy=True) for k in ('positions', 'velocities', 'densities', 'masses',
                                                                    'isFluid')}
    stepper = stepperFor(case)
    for _ in range(steps):
        stepper(ref)
    assertFollows(out, time, ref, stepper.time)


def test_the_refined_ridge_follows_the_oracle():
    # the device's crest-zone split (every fluid particle under a surface 0.3 H above still water, into 8
    # daughters of h / 2), then mixed-h steps on the device and in float64 from the split state
    case = shortRidge()
    sums = cases.pairSumsFor(case)
    state = case.state.copy()
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    before = sums.pullState()
    split = cases.refineCrestZone(sums, case, lengthRatio=0.5)
    assert split > 0
    start = sums.pullState()
    assert start['masses'].sum() == pytest.approx(before['masses'].sum(), rel=1e-15)
    steps = 20
    shortest = float(start['lengths'].min())
    time, step, _ = sums.advance(0.0, 0, math.inf, steps, shortest, case.cflNumber, case.maxTimeStep)
    assert step == steps
    out = sums.pullState()
    ref = {k: start[k].copy() for k in ('positions', 'velocities', 'densities', 'masses', 'isFluid', 'lengths')}
    stepper = stepperFor(case)
    for _ in range(steps):
        stepper(ref)
    assertFollows(out, time, ref, stepper.time)
