"""Two levels of smoothing length: the fine grid the split particles are sorted into.

A particle shorter than the grid's h (a split's daughter) is sorted into a second grid sized for the
fine level, and every particle searches each grid only as far as that grid's particles reach
(src/pysurf/sphGpu.py:52-56, 331-363: reach h_i + h_max, h_ij the mean).  The candidates each search
offers are a superset of the pairs, so the sums and their order are the walk's whichever way the
neighbours are found; these tests hold the two-level walk to the reference's rows and the oracle.
"""
import math

import numpy as np
import pytest

from conftest import golden
from pysurf_b200 import cases
from test_gpu_steps import deviceRun

pytestmark = pytest.mark.gpu

CLOUDS = ['2d_o_cubicSpline', '3d_o_wendlandC2', '3d_p_cubicSpline']


@pytest.mark.parametrize('tag', CLOUDS)
def test_neighbour_rows_are_the_references_with_two_levels(tag):
    # the reference's compressed rows (src/pysurf/sphCompiled.py:133-234) depend on the positions only:
    # giving half the particles h / 2 moves them to the fine grid and must change no row
    from pysurf_b200.sphGpu import PairSums
    c = golden('clouds.npz', tag)
    x = c['positions']
    h = float(c['h'])
    lengths = h * np.random.default_rng(5).choice([1.0, 0.5], size=len(c['masses']))
    kernelType = 'wendlandC2' if int(c['kernel']) == 1 else 'cubicSpline'
    s = PairSums(x.shape[1], h, x.min(axis=0), x.max(axis=0), float(c['period']), device='cuda:0',
                 kernelType=kernelType)
    s.update(x, c['masses'], c['isFluid'], lengths)
    offsets, neighbors = s.neighborList(2.0 * h)
    assert np.array_equal(np.diff(offsets), np.diff(c['offsets']))
    for i in range(len(offsets) - 1):
        mine = np.sort(neighbors[offsets[i]:offsets[i + 1]])
        theirs = np.sort(c['neighbors'][c['offsets'][i]:c['offsets'][i + 1]])
        assert np.array_equal(mine, theirs), i


def splitBeach():
    case = cases.solitaryBeach(particlesPerDepth=8)
    state = case.state.copy()
    crest = state.isFluid & (state.positions[:, 0] > 8.0) & (state.positions[:, 0] < 12.0)
    return case, state, crest


@pytest.mark.parametrize('threads', [1, 4])
def test_the_table_changes_no_bit_with_two_levels(threads):
    # the table records the two-level walk's order, so a split run's bits are the walk's
    runs = []
    for table in (False, True):
        case, state, crest = splitBeach()
        sums = cases.pairSumsFor(case)
        sums.setSweepOptions(table, threads)
        sums.push(state)
        sums.setBoundary(case.boundary, state)
        sums.split(crest, case.referenceDensity, 0.5)
        shortest = float(sums.pullState()['lengths'].min())
        sums.advance(0.0, 0, math.inf, 20, shortest, case.cflNumber, case.maxTimeStep)
        runs.append(sums.pullState())
    for name in ('positions', 'velocities', 'densities'):
        assert np.array_equal(runs[0][name], runs[1][name]), name


def test_a_second_split_level_steps_like_the_oracle():
    # daughters split again (h / 4) share the fine grid with their h / 2 cousins
    from oracle import oracle
    case, state, crest = splitBeach()
    sums = cases.pairSumsFor(case)
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    sums.split(crest, case.referenceDensity, 0.5)
    once = sums.pullState()
    inner = once['isFluid'] & (once['positions'][:, 0] > 9.5) & (once['positions'][:, 0] < 10.5)
    sums.split(inner, case.referenceDensity, 0.5)
    split = sums.pullState()
    assert np.isclose(split['lengths'].min(), 0.25 * case.smoothingLength)
    shortest = float(split['lengths'].min())
    time, step, dt = sums.advance(0.0, 0, math.inf, 15, shortest, case.cflNumber, case.maxTimeStep)
    out = sums.pullState()
    ref = {k: split[k].copy() for k in ('positions', 'velocities', 'densities', 'masses', 'isFluid', 'lengths')}
    stepper = oracle.Stepper(2, case.kernelType, case.smoothingLength, case.referenceDensity, case.soundSpeed,
                             case.alpha, case.gravity, 0.0, 0.0, case.densityFloor, case.densityDiffusion, 0.1, True,
                             False, True, True, case.cflNumber, case.maxTimeStep, 0.0, 0,
                             ('bed', oracle.bedParams(case.boundary.bathymetry.x, case.boundary.bathymetry.z,
                                                      0.25 * case.spacing, False, 0.0, True, 0.0, 0.0,
                                                      case.boundary.bathymetry.endX)))
    for _ in range(15):
        stepper(ref)
    assert time == pytest.approx(stepper.time, rel=1e-4)
    assert np.abs(out['positions'] - ref['positions']).max() < 1e-6
    assert np.abs(out['velocities'] - ref['velocities']).max() < 1e-3
