"""Device-resident steps against the reference's own float64 host steps and the float64 oracle.

The runs are the reference's numpy solver stepping the sloshing tank of tests/testSphGpu.py:441-457
under each scheme, and a solitary wave over a bed under the deltaSph scheme (tests/golden/runs.npz).
Tolerances are those the reference holds its float32 device to against the numpy solver
(tests/testSphGpu.py:503-517, 578-590): positions 1e-6 m, velocities and densities 1e-3, time 1e-4.
"""
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden, goldenTags
from oracle import oracle
from pysurf_b200 import cases
from pysurf_b200.state import BedBoundary, ContainerBoundary, ParticleState, Profile

pytestmark = pytest.mark.gpu

RUNS = goldenTags('runs.npz')
MODES = ['none', 'molteni', 'hydrostatic', 'antuono']


def caseFromRun(r) -> cases.Case:
    (dim, kind, h, rho0, c0, alpha, bf, xsph, floor, mode, delta, wall, tension, corrected, limited, cfl, maxdt,
     interval, period) = r['config']
    n = len(r['masses'])
    state = ParticleState(r['positions'].copy(), r['velocities'].copy(), np.zeros_like(r['positions']),
                          r['densities'].copy(), np.zeros(n), r['masses'].copy(), r['isFluid'].copy())
    if int(r['boundary_kind']) == 1:
        boundary = ContainerBoundary(r['boundary_lower'], r['boundary_upper'], 0.005, 3, bool(r['boundary_openTop']))
    else:
        clearance, side, width, offshore, wallX, piston, endLimit = r['boundary_params']
        profile = Profile(r['boundary_bedX'], r['boundary_bedZ'], 1.0)
        boundary = BedBoundary(profile, 4.0 * clearance, 6, wallTop=1.9 if offshore else None, width=None,
                               endWallTop=1.9 if endLimit < profile.endX else None, wallX=wallX)
    domain = r['domain']
    return cases.Case('run', state, boundary, int(dim), 0.0, h, 'wendlandC2' if int(kind) == 1 else 'cubicSpline',
                      domain[0], domain[1], rho0, c0, r['gravity'], alpha=alpha, boundaryViscosityFactor=bf,
                      xsphEpsilon=xsph, densityFloor=floor, densityDiffusion=MODES[int(mode)], diffusionDelta=delta,
                      wallExtrapolated=bool(wall), negativePressure=bool(tension), continuityCorrection=bool(corrected),
                      viscosityLimiter=bool(limited), cflNumber=cfl, maxTimeStep=maxdt,
                      densityFilterInterval=int(interval), period=period)


def deviceRun(case, steps, cellsPerSupport=None, table=True, threads=None):
    # threads None keeps the backend's default, which hostDrivenRun's PairSums also runs with
    sums = cases.pairSumsFor(case, cellsPerSupport)
    if threads is not None or not table:
        sums.setSweepOptions(table, threads or 4)
    state = case.state.copy()
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    time, step, dt = sums.advance(0.0, 0, math.inf, steps, case.smoothingLength, case.cflNumber, case.maxTimeStep,
                                  case.densityFilterInterval)
    assert step == steps
    sums.pull(state)
    return state, time, sums


def hostDrivenRun(case, steps):
    # the reference's own loop: residentRates, the host's cflTimeStep, residentIntegrate (src/pysurf/sphSolver.py:1980-1989)
    sums = cases.pairSumsFor(case)
    state = case.state.copy()
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    time = 0.0
    interval = case.densityFilterInterval
    for k in range(steps):
        vmax, amax = sums.residentRates(bool(interval) and k > 0 and k % interval == 0)
        dt = case.cflNumber * case.smoothingLength / (case.soundSpeed + vmax)
        if amax > 1e-12:
            dt = min(dt, case.cflNumber * math.sqrt(case.smoothingLength / amax))
        dt = min(dt, case.maxTimeStep)
        sums.residentIntegrate(dt)
        time += dt
    sums.pull(state)
    return state, time


@pytest.mark.parametrize('tag', RUNS)
def test_device_steps_follow_the_reference_host_steps(tag):
    r = golden('runs.npz', tag)
    case = caseFromRun(r)
    steps = int(r['steps'])
    state, time, _ = deviceRun(case, steps)
    assert time == pytest.approx(float(np.sum(r['dts'])), rel=1e-4)
    assert np.abs(state.positions - r['finalPositions']).max() < 1e-6
    assert np.abs(state.velocities - r['finalVelocities']).max() < 1e-3
    assert np.abs(state.densities - r['finalDensities']).max() < 1e-3


@pytest.mark.parametrize('tag', RUNS)
def test_device_steps_follow_the_oracle(tag):
    r = golden('runs.npz', tag)
    case = caseFromRun(r)
    steps = int(r['steps'])
    state, time, _ = deviceRun(case, steps)
    boundary = ('container', r['boundary_lower'], r['boundary_upper'], True) if int(r['boundary_kind']) == 1 else (
        'bed', oracle.bedParams(r['boundary_bedX'], r['boundary_bedZ'], *r['boundary_params']))
    stepper = oracle.Stepper(case.dimensions, case.kernelType, case.smoothingLength, case.referenceDensity,
                             case.soundSpeed, case.alpha, case.gravity, case.boundaryViscosityFactor, case.xsphEpsilon,
                             case.densityFloor, case.densityDiffusion, case.diffusionDelta, case.wallExtrapolated,
                             case.negativePressure, case.continuityCorrection, case.viscosityLimiter, case.cflNumber,
                             case.maxTimeStep, 0.0, case.densityFilterInterval, boundary)
    ref = {k: r[k].copy() for k in ('positions', 'velocities', 'densities', 'masses', 'isFluid')}
    for _ in range(steps):
        stepper(ref)
    assert time == pytest.approx(stepper.time, rel=1e-4)
    assert np.abs(state.positions - ref['positions']).max() < 1e-6
    assert np.abs(state.velocities - ref['velocities']).max() < 1e-3
    assert np.abs(state.densities - ref['densities']).max() < 1e-3


@pytest.mark.parametrize('tag', ['plain', 'deltaHydrostatic', 'bedDelta'])
def test_the_device_loop_is_the_host_loop_bit_for_bit(tag):
    # the time step taken on the device is the host's cflTimeStep to the last bit, so the two loops agree exactly
    case = caseFromRun(golden('runs.npz', tag))
    device, deviceTime, _ = deviceRun(case, 35)
    host, hostTime = hostDrivenRun(case, 35)
    assert deviceTime == hostTime
    assert np.array_equal(device.positions, host.positions)
    assert np.array_equal(device.velocities, host.velocities)
    assert np.array_equal(device.densities, host.densities)


def test_a_resumed_run_follows_the_uninterrupted_one_bit_for_bit():
    # tests/testBreakingWave3D.py:270-296: the sums run in a fixed order, so a run pulled to the host and pushed
    # back continues exactly as one that never stopped
    case = caseFromRun(golden('runs.npz', 'bedDelta'))
    whole, wholeTime, _ = deviceRun(case, 40)
    sums = cases.pairSumsFor(case)
    state = case.state.copy()
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    time, step, dt = sums.advance(0.0, 0, math.inf, 17, case.smoothingLength, case.cflNumber, case.maxTimeStep)
    sums.pull(state)
    sums2 = cases.pairSumsFor(case)
    sums2.push(state)
    sums2.setBoundary(case.boundary, state)
    time, step, dt = sums2.advance(time, step, math.inf, 40, case.smoothingLength, case.cflNumber, case.maxTimeStep,
                                   0, dt)
    sums2.pull(state)
    assert step == 40 and time == wholeTime
    assert np.array_equal(state.positions, whole.positions)
    assert np.array_equal(state.velocities, whole.velocities)
    assert np.array_equal(state.densities, whole.densities)


def test_cell_size_changes_only_the_order_of_sums():
    # the cell list's resolution changes which cells are walked and the order neighbours are summed in
    # (the sort is by cell, then index), not the pairs: the runs agree to float32 rounding of the sums
    case = caseFromRun(golden('runs.npz', 'deltaWendland'))
    a, ta, _ = deviceRun(case, 20, cellsPerSupport=1)
    b, tb, _ = deviceRun(case, 20, cellsPerSupport=2)
    assert abs(ta - tb) <= 1e-9 * ta
    assert np.abs(a.positions - b.positions).max() < 1e-9
    assert np.abs(a.velocities - b.velocities).max() < 1e-5


@pytest.mark.parametrize('mode', ['hydrostatic', 'antuono'])
def test_a_delta_sph_still_tank_stays_at_rest(mode):
    # tests/testSphGpu.py:549-575: max |v| < 0.01 sqrt(g d) and drift < 0.25 dx over 0.2 s
    case = cases.sloshingTank(tilt=0.0, densityFilterInterval=0, xsphEpsilon=0.0, wallExtrapolated=True,
                              continuityCorrection=True, densityFloor=0.9, densityDiffusion=mode)
    sums = cases.pairSumsFor(case)
    state = case.state.copy()
    start = state.positions[state.isFluid].copy()
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    time, step, dt = sums.advance(0.0, 0, 0.2, 1 << 40, case.smoothingLength, case.cflNumber, case.maxTimeStep)
    sums.pull(state)
    assert time >= 0.2
    fill = case.info['fillHeight']
    speed = np.linalg.norm(state.velocities[state.isFluid], axis=1).max()
    assert speed < 0.01 * math.sqrt(cases.GRAVITY * fill)
    assert np.abs(state.positions[state.isFluid] - start).max() < 0.25 * case.spacing


def test_mass_is_conserved_exactly_through_a_split():
    # src/pysurf/sphRefinement.py:136-190 on the device against the oracle's restatement of it
    case = cases.solitaryBeach(particlesPerDepth=8)
    sums = cases.pairSumsFor(case)
    state = case.state.copy()
    sums.push(state)
    rng = np.random.default_rng(3)
    mask = (rng.uniform(size=state.nParticles) < 0.2)
    for ratio in (1.0, 0.5):
        sums = cases.pairSumsFor(case)
        sums.push(state)
        count = sums.split(mask, case.referenceDensity, ratio)
        out = sums.pullState()
        expected = {k: np.array(getattr(state, k), copy=True) for k in ('positions', 'velocities', 'densities',
                                                                          'masses', 'isFluid')}
        expected['lengths'] = np.full(state.nParticles, case.smoothingLength)
        assert count == oracle.splitParticles(expected, mask, case.referenceDensity, case.smoothingLength, ratio)
        assert np.array_equal(out['masses'], expected['masses'])
        assert np.array_equal(out['isFluid'], expected['isFluid'])
        assert np.allclose(out['positions'], expected['positions'], rtol=0.0, atol=1e-14)
        assert np.array_equal(out['velocities'], expected['velocities'])
        assert np.array_equal(out['densities'], expected['densities'])
        assert np.array_equal(out['lengths'], expected['lengths'])
        assert out['masses'].sum() == pytest.approx(state.masses.sum(), rel=1e-15)


def test_a_split_beach_steps_like_the_oracle():
    # mixed smoothing lengths (h halved in the split zone) stepped on the device and in float64
    case = cases.solitaryBeach(particlesPerDepth=8)
    state = case.state.copy()
    crest = state.isFluid & (state.positions[:, 0] > 8.0) & (state.positions[:, 0] < 12.0)
    sums = cases.pairSumsFor(case)
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    sums.split(crest, case.referenceDensity, 0.5)
    split = sums.pullState()
    minLength = float(split['lengths'].min())
    time, step, dt = sums.advance(0.0, 0, math.inf, 25, minLength, case.cflNumber, case.maxTimeStep)
    out = sums.pullState()
    ref = {k: split[k].copy() for k in ('positions', 'velocities', 'densities', 'masses', 'isFluid', 'lengths')}
    stepper = oracle.Stepper(2, case.kernelType, case.smoothingLength, case.referenceDensity, case.soundSpeed,
                             case.alpha, case.gravity, 0.0, 0.0, case.densityFloor, case.densityDiffusion, 0.1, True,
                             False, True, True, case.cflNumber, case.maxTimeStep, 0.0, 0,
                             ('bed', oracle.bedParams(case.boundary.bathymetry.x, case.boundary.bathymetry.z,
                                                      0.25 * case.spacing, False, 0.0, True, 0.0, 0.0,
                                                      case.boundary.bathymetry.endX)))
    for _ in range(25):
        stepper(ref)
    assert time == pytest.approx(stepper.time, rel=1e-4)
    assert np.abs(out['positions'] - ref['positions']).max() < 1e-6
    assert np.abs(out['velocities'] - ref['velocities']).max() < 1e-3


@pytest.mark.parametrize('tag', ['plain', 'deltaWendland', 'bedDelta'])
def test_the_neighbour_table_changes_no_bit(tag):
    # the table keeps the cell walk's order, so the sums, and the whole run, are the same bits
    case = caseFromRun(golden('runs.npz', tag))
    walked, tw, _ = deviceRun(case, 25, table=False)
    listed, tl, _ = deviceRun(case, 25, table=True)
    assert tw == tl
    assert np.array_equal(walked.positions, listed.positions)
    assert np.array_equal(walked.velocities, listed.velocities)
    assert np.array_equal(walked.densities, listed.densities)


@pytest.mark.parametrize('threads', [2, 4, 8])
@pytest.mark.parametrize('table', [True, False])
@pytest.mark.parametrize('tag', ['deltaWendland', 'bedDelta', 'limited'])
def test_threads_per_particle_follow_the_reference(tag, table, threads):
    # several threads to a particle change only the order of the float32 sums
    r = golden('runs.npz', tag)
    case = caseFromRun(r)
    steps = int(r['steps'])
    state, time, _ = deviceRun(case, steps, table=table, threads=threads)
    assert time == pytest.approx(float(np.sum(r['dts'])), rel=1e-4)
    assert np.abs(state.positions - r['finalPositions']).max() < 1e-6
    assert np.abs(state.velocities - r['finalVelocities']).max() < 1e-3
    assert np.abs(state.densities - r['finalDensities']).max() < 1e-3


def test_threads_per_particle_on_the_benchmark_beach():
    # the 64-ppd beach (122k particles) five steps at one and eight threads a particle: the same run to
    # float32 rounding of the sums (a grid eight times longer must find room for every block's maxima)
    case = cases.solitaryBeach(particlesPerDepth=64)
    runs = []
    for threads in (1, 8):
        sums = cases.pairSumsFor(case)
        sums.setSweepOptions(True, threads)
        state = case.state.copy()
        sums.push(state)
        sums.setBoundary(case.boundary, state)
        time, step, dt = sums.advance(0.0, 0, math.inf, 5, case.smoothingLength, case.cflNumber, case.maxTimeStep)
        sums.pull(state)
        runs.append((time, state))
    (t1, a), (t8, b) = runs
    assert t8 == pytest.approx(t1, rel=1e-9)
    assert np.abs(a.positions - b.positions).max() < 1e-9
    assert np.abs(a.velocities - b.velocities).max() < 1e-5


def test_the_closure_run_follows_the_reference_host_steps():
    # a sloshing tank under the delta-LES-SPH closure (turbulenceClosure 'deltaLes'), 30 device steps
    # against the reference's float64 host steps and the oracle's
    r = golden('closure.npz', 'closure')
    case = caseFromRun(r)
    case.turbulenceClosure = 'deltaLes'
    case.kinematicViscosity = float(np.load(os.path.join(GOLDEN, 'closure.npz'))['viscosity'])
    steps = int(r['steps'])
    state, time, _ = deviceRun(case, steps)
    assert time == pytest.approx(float(np.sum(r['dts'])), rel=1e-4)
    assert np.abs(state.positions - r['finalPositions']).max() < 1e-6
    assert np.abs(state.velocities - r['finalVelocities']).max() < 1e-3
    assert np.abs(state.densities - r['finalDensities']).max() < 1e-3


def test_the_shifting_run_follows_the_reference_host_steps():
    # a sloshing tank with particle shifting, 30 device steps against the reference's float64 host
    # steps and the oracle's
    data = np.load(os.path.join(GOLDEN, 'shifting.npz'))
    r = golden('shifting.npz', 'shifting')
    case = caseFromRun(r)
    case.particleShifting = True
    case.shiftingMach = float(data['shifting/mach'])
    case.spacing = float(data['shifting/spacing'])
    steps = int(r['steps'])
    state, time, _ = deviceRun(case, steps)
    assert time == pytest.approx(float(np.sum(r['dts'])), rel=1e-4)
    assert np.abs(state.positions - r['finalPositions']).max() < 1e-6
    assert np.abs(state.velocities - r['finalVelocities']).max() < 1e-3
    assert np.abs(state.densities - r['finalDensities']).max() < 1e-3


@pytest.mark.parametrize('steps', [100, 1000])
def test_the_dam_break_follows_the_oracle(steps):
    # the CPU-runnable dam break: the 1 x 2 m column in the 4 x 3 m tank at 0.02 m (5,000 fluid particles,
    # jittered from seed 0), Wendland C2 at h = 1.3 dx, hydrostatic delta-SPH, device steps against the
    # float64 oracle's: 100, and the 1,000 the benchmark configuration runs
    from oracle import oracle
    case = cases.damBreak()
    state, time, _ = deviceRun(case, steps)
    b = case.boundary
    stepper = oracle.Stepper(2, case.kernelType, case.smoothingLength, case.referenceDensity, case.soundSpeed,
                             case.alpha, case.gravity, case.boundaryViscosityFactor, case.xsphEpsilon,
                             case.densityFloor, case.densityDiffusion, case.diffusionDelta, case.wallExtrapolated,
                             case.negativePressure, case.continuityCorrection, case.viscosityLimiter, case.cflNumber,
                             case.maxTimeStep, 0.0, case.densityFilterInterval,
                             ('container', b.containerMin, b.containerMax, b.openTop))
    ref = {k: np.array(getattr(case.state, k), copy=True) for k in ('positions', 'velocities', 'densities', 'masses',
                                                                    'isFluid')}
    for _ in range(steps):
        stepper(ref)
    errors = (abs(time - stepper.time) / stepper.time, np.abs(state.positions - ref['positions']).max(),
              np.abs(state.velocities - ref['velocities']).max(), np.abs(state.densities - ref['densities']).max())
    print(f'\ndam break, {steps} steps to t = {stepper.time:.4f} s: time {errors[0]:.1e} relative, positions '
          f'{errors[1]:.1e} m, velocities {errors[2]:.1e} m/s, densities {errors[3]:.1e} kg/m^3')
    assert errors[0] < 1e-5
    assert errors[1] < 1e-6
    assert errors[2] < 1e-3
    assert errors[3] < 1e-2
