"""Momentum and continuity sums against the float64 oracle, compensated and plain.

Each particle's du/dt and drho/dt on the 32- and 64-ppd beaches (about 110 neighbours a particle) and on the
golden clouds, and whole device runs, are compared with the oracle's float64 results; the error of
each is stated (run with -s to print it) and held to the reference's criterion for its float32
device, 1e-5 of the largest value (tests/testSphGpu.py:79-404).
"""
import math

import numpy as np
import pytest

from conftest import golden, goldenTags
from oracle import oracle
from pysurf_b200 import cases
from pysurf_b200._lib import SphError

pytestmark = pytest.mark.gpu

CLOUDS = goldenTags('clouds.npz')


def relativeError(result, expected) -> float:
    return float(np.abs(result - expected).max() / np.abs(expected).max())


def beachSums(case, compensated):
    from pysurf_b200.sphGpu import PairSums
    st = case.state
    s = PairSums(case.dimensions, case.smoothingLength, case.domainMin, case.domainMax, 0.0, device='cuda:0',
                 kernelType=case.kernelType)
    s.setCompensatedSums(compensated)
    s.update(st.positions, st.masses, st.isFluid)
    return s


@pytest.mark.parametrize('particlesPerDepth', [32, 64])
def test_beach_rates_against_the_oracle(particlesPerDepth):
    case = cases.solitaryBeach(particlesPerDepth=particlesPerDepth)
    st = case.state
    rho0, c0 = case.referenceDensity, case.soundSpeed
    pressures = rho0 * c0 * c0 / 7.0 * ((st.densities / rho0) ** 7 - 1.0)
    o = oracle.System(st.positions, st.masses, st.isFluid, np.full(st.nParticles, case.smoothingLength),
                      case.kernelType, 0.0)
    g = case.gravity
    expectedA = o.pairAccelerations(st.velocities, st.densities, pressures, c0, case.alpha, 1.0, g)
    L = o.correctionMatrices(st.densities)
    expectedR = o.continuityRate(st.velocities, st.densities, 'hydrostatic', case.diffusionDelta, c0, rho0,
                                 abs(float(g[-1])), corrections=L)
    errors, results = {}, {}
    fluid = st.isFluid
    for compensated in (False, True):
        s = beachSums(case, compensated)
        a = s.pairAccelerations(st.velocities, st.densities, pressures, c0, case.alpha, 1.0, g)
        s.setDiffusion('hydrostatic', case.diffusionDelta, c0, rho0, abs(float(g[-1])))
        s.setContinuityCorrection(True)
        r = s.continuityRate(st.velocities, st.densities)
        scale = np.abs(expectedR).max()
        errors[compensated] = (relativeError(a[fluid], expectedA[fluid]), relativeError(r, expectedR),
                               float(np.abs(r - expectedR)[fluid].max() / scale),
                               float(np.abs(r - expectedR)[~fluid].max() / scale))
        results[compensated] = (a, r)
    for compensated, e in errors.items():
        print(f'\n{particlesPerDepth}-ppd beach, {st.nParticles} particles, {"compensated" if compensated else "plain"} sums: '
              f'du/dt error {e[0]:.2e} of the largest value; drho/dt {e[1]:.2e} (fluid rows {e[2]:.2e}, '
              f'boundary rows {e[3]:.2e})')
    # Both within the reference's 1e-5 of the largest value.  The start is near hydrostatic rest, where
    # the hydrostatic diffusion's difference nearly cancels: the frame's deviation remainders and the
    # split subtraction keep that difference's float64 digits, so drho/dt meets it too.  Compensation
    # removes the sum's own share of du/dt's error; the sums are deterministic, so that holds run to run.
    for e in errors.values():
        assert e[0] <= 1e-5 and e[1] <= 1e-5
    assert errors[True][0] <= errors[False][0]
    # the switch reaches the sums
    assert not np.array_equal(results[False][0], results[True][0])
    assert not np.array_equal(results[False][1], results[True][1])


@pytest.mark.parametrize('tag', CLOUDS)
def test_compensated_cloud_sums_keep_the_references_tolerance(tag):
    c = golden('clouds.npz', tag)
    from pysurf_b200.sphGpu import PairSums
    x = c['positions']
    dim = x.shape[1]
    g = np.zeros(dim)
    g[-1] = -9.81
    kernelType = 'wendlandC2' if int(c['kernel']) == 1 else 'cubicSpline'
    s = PairSums(dim, float(c['h']), x.min(axis=0), x.max(axis=0), float(c['period']), device='cuda:0',
                 kernelType=kernelType)
    s.setCompensatedSums(True)
    s.update(x, c['masses'], c['isFluid'])
    a = s.pairAccelerations(c['velocities'], c['densities'], c['pressures'], 20.0, 0.1, 0.3, g)
    assert relativeError(a, c['accelerations']) <= 1e-5
    assert relativeError(s.continuityRate(c['velocities']), c['continuity']) <= 1e-5
    s.setDiffusion('hydrostatic', 0.1, 20.0, 1000.0, 9.81)
    assert relativeError(s.continuityRate(c['velocities'], c['densities']), c['diffusive_hydrostatic']) <= 1e-5


def test_a_compensated_beach_run_follows_the_plain_one_and_refuses_the_energy_budget():
    case = cases.solitaryBeach(particlesPerDepth=16)
    runs = []
    for compensated in (False, True):
        sums = cases.pairSumsFor(case)
        sums.setCompensatedSums(compensated)
        state = case.state.copy()
        sums.push(state)
        sums.setBoundary(case.boundary, state)
        t, step, _ = sums.advance(0.0, 0, math.inf, 100, case.smoothingLength, case.cflNumber, case.maxTimeStep,
                                  case.densityFilterInterval)
        assert step == 100
        sums.pull(state)
        runs.append((t, state))
        if compensated:
            with pytest.raises(SphError):
                sums.setEnergyBudget(True)
            sums.setCompensatedSums(False)
            sums.setEnergyBudget(True)
            with pytest.raises(SphError):
                sums.setCompensatedSums(True)
    (t0, a), (t1, b) = runs
    assert t1 == pytest.approx(t0, rel=1e-5)
    assert np.abs(a.positions - b.positions).max() < 1e-5
    assert np.abs(a.velocities - b.velocities).max() < 1e-3
    assert np.abs(a.densities - b.densities).max() < 1e-3
    assert not np.array_equal(a.densities, b.densities)
