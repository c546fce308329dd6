"""The merge on the device against the reference's merges (tests/golden/merge.npz), and a run that
splits, steps, merges and steps again against the oracle doing the same."""
import math

import numpy as np
import pytest

from pysurf_b200 import cases
from pysurf_b200.state import ParticleState
from test_merge_oracle import FIELDS, MERGE, TAGS

pytestmark = pytest.mark.gpu


def pushed(tag):
    from pysurf_b200.sphGpu import PairSums
    state = ParticleState(*(MERGE[f'{tag}/{name}'].copy() for name in FIELDS))
    rho0, referenceMass, length, ratio = MERGE[f'{tag}/reference']
    x = state.positions
    sums = PairSums(x.shape[1], float(length), x.min(axis=0) - 0.1, x.max(axis=0) + 0.1, device='cuda:0')
    sums.push(state)
    return sums, (rho0, referenceMass, length, ratio)


@pytest.mark.parametrize('tag', TAGS)
def test_the_device_merges_as_the_reference(tag):
    sums, (rho0, referenceMass, length, ratio) = pushed(tag)
    groups, removed, source = sums.merge(MERGE[f'{tag}/mask'], rho0, referenceMass, ratio)
    assert groups == int(MERGE[f'{tag}/groups'])
    assert np.array_equal(source, MERGE[f'{tag}/source'])
    assert removed == pytest.approx(float(MERGE[f'{tag}/removedEnergy']), rel=1e-12)
    after = sums.pullState()
    for name in ('masses', 'isFluid', 'lengths'):
        assert np.array_equal(after[name], MERGE[f'{tag}/merged_{name}']), name
    # the group sums' order may differ from numpy's einsum by a rounding
    for name in ('positions', 'velocities', 'densities'):
        assert np.allclose(after[name], MERGE[f'{tag}/merged_{name}'], rtol=1e-14, atol=1e-14), name


def test_nothing_merges_when_nothing_split():
    tag = TAGS[0]
    sums, (rho0, referenceMass, length, ratio) = pushed(tag)
    before = sums.pullState()
    fluid = MERGE[f'{tag}/isFluid']
    unsplit = fluid & (MERGE[f'{tag}/masses'] >= referenceMass * (1.0 - 1e-12))
    groups, removed, source = sums.merge(unsplit, rho0, referenceMass, ratio)
    assert groups == 0 and removed == 0.0 and np.array_equal(source, np.arange(len(fluid)))
    after = sums.pullState()
    for name in ('positions', 'velocities', 'masses'):
        assert np.array_equal(after[name], before[name])


def test_the_energy_budget_carries_its_totals_through_a_merge():
    # the merged-away members' running totals join their group's, so the sums hold across the merge
    case = cases.solitaryBeach(particlesPerDepth=8)
    case.trackEnergy = True
    state = case.state.copy()
    crest = state.isFluid & (state.positions[:, 0] > 8.0) & (state.positions[:, 0] < 12.0)
    sums = cases.pairSumsFor(case)
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    sums.split(crest, case.referenceDensity, 0.5)
    sums.advance(0.0, 0, math.inf, 10, 0.5 * case.smoothingLength, case.cflNumber, case.maxTimeStep)
    before = sums.energySums()
    referenceMass = float(np.max(state.masses[state.isFluid]))
    groups, _, _ = sums.merge(np.ones(sums.count, dtype=bool), case.referenceDensity, referenceMass, 0.5)
    assert groups > 0
    assert np.allclose(sums.energySums(), before, rtol=1e-12, atol=1e-15 * np.abs(before).sum())


def test_a_split_step_merge_step_run_follows_the_oracle():
    from oracle import oracle
    case = cases.solitaryBeach(particlesPerDepth=8)
    state = case.state.copy()
    crest = state.isFluid & (state.positions[:, 0] > 8.0) & (state.positions[:, 0] < 12.0)
    referenceMass = float(np.max(state.masses[state.isFluid]))
    sums = cases.pairSumsFor(case)
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    sums.split(crest, case.referenceDensity, 0.5)
    ref = {k: v.copy() for k, v in sums.pullState().items()}
    shortest = 0.5 * case.smoothingLength
    time, step, dt = sums.advance(0.0, 0, math.inf, 10, shortest, case.cflNumber, case.maxTimeStep)
    after = sums.pullState()
    behind = after['isFluid'] & (after['positions'][:, 0] < 10.0)
    groups, removed, source = sums.merge(behind, case.referenceDensity, referenceMass, 0.5)
    assert groups > 0
    merged = sums.pullState()
    shortest = float(merged['lengths'].min())
    time, step, dt = sums.advance(time, step, math.inf, 20, shortest, case.cflNumber, case.maxTimeStep, 0, dt)
    out = sums.pullState()

    stepper = oracle.Stepper(2, case.kernelType, case.smoothingLength, case.referenceDensity, case.soundSpeed,
                             case.alpha, case.gravity, 0.0, 0.0, case.densityFloor, case.densityDiffusion, 0.1, True,
                             False, True, True, case.cflNumber, case.maxTimeStep, 0.0, 0,
                             ('bed', oracle.bedParams(case.boundary.bathymetry.x, case.boundary.bathymetry.z,
                                                      0.25 * case.spacing, False, 0.0, True, 0.0, 0.0,
                                                      case.boundary.bathymetry.endX)))
    for _ in range(10):
        stepper(ref)
    # the same mask (caller order is shared); the groups agree unless a position lies within the
    # runs' 1e-7 m of a cube's face
    hostGroups, hostRemoved, hostSource = oracle.mergeParticles(ref, behind, case.referenceDensity, referenceMass,
                                                                case.smoothingLength, 0.5)
    assert hostGroups == groups and np.array_equal(hostSource, source)
    for _ in range(10):
        stepper(ref)
    assert time == pytest.approx(stepper.time, rel=1e-4)
    assert np.abs(out['positions'] - ref['positions']).max() < 1e-6
    assert np.abs(out['velocities'] - ref['velocities']).max() < 1e-3


def test_a_merge_that_cannot_fill_the_boundarys_places_fails_and_changes_nothing():
    # src/pysurf/sphRefinement.py:296-297 raises when too few fluid particles follow the boundary to
    # fill the places a merge leaves among it; here every daughter stands before the boundary
    from pysurf_b200 import _lib
    from pysurf_b200.sphGpu import PairSums
    s, rho0 = 0.05, 1000.0
    referenceMass = rho0 * s * s
    axes = np.arange(16) * 0.5 * s + 0.25 * s
    daughters = np.stack(np.meshgrid(axes, axes, indexing='ij'), axis=-1).reshape(-1, 2) + 0.3
    wall = np.stack([np.linspace(0.0, 1.5, 40), np.zeros(40)], axis=1)
    n = len(daughters) + len(wall)
    state = ParticleState(np.vstack([daughters, wall]), np.zeros((n, 2)), np.zeros((n, 2)), np.full(n, rho0),
                          np.zeros(n), np.full(n, referenceMass / 4), np.r_[np.ones(len(daughters), bool),
                                                                           np.zeros(len(wall), bool)],
                          np.full(n, 0.65 * s))
    x = state.positions
    sums = PairSums(2, 1.3 * s, x.min(axis=0) - 0.1, x.max(axis=0) + 0.1, device='cuda:0')
    sums.push(state)
    before = sums.pullState()
    with pytest.raises(_lib.SphError):
        sums.merge(np.ones(n, dtype=bool), rho0, referenceMass, 0.5)
    after = sums.pullState()
    assert sums.count == n
    for name in ('positions', 'velocities', 'densities', 'masses', 'lengths', 'isFluid'):
        assert np.array_equal(after[name], before[name]), name
