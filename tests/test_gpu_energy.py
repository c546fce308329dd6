"""The energy budget on the device against the reference's own budgets (tests/golden/energy.npz).

The fixtures are the reference array solver's budgets over its energy runs (tests/testSphEnergy.py)
and over sloshing runs that reach the filter, wall viscosity, shifting, the clamp and the floor; the
oracle restates them to 1e-9 of the terms' throughput (tests/test_energy_oracle.py).  The device sums
its parts in float32 and integrates the state in float64, so its terms follow the reference's to
1e-3 of the throughput and close on the change of the fluid's energy to 1e-5 of it, the reference's
own bars for its device budget (tests/testSphEnergy.py:189-241).
"""
import math

import numpy as np
import pytest

from conftest import golden
from pysurf_b200 import cases
from pysurf_b200.sphGpu import energyTerms
from test_gpu_steps import caseFromRun

pytestmark = pytest.mark.gpu

RUNS = ['channel', 'uncorrected', 'published', 'hybrid', 'filtered', 'shifted', 'clamped']


def budgetCase(tag, track=True):
    r = golden('energy.npz', tag)
    case = caseFromRun(r)
    case.turbulenceClosure = 'deltaLes' if int(r['closure']) else 'none'
    case.particleShifting = bool(r['shifting'][0])
    case.shiftingMach, case.spacing = float(r['shifting'][1]), float(r['shifting'][2])
    case.trackEnergy = track
    return r, case


def run(case, steps, spans=1):
    sums = cases.pairSumsFor(case)
    state = case.state.copy()
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    start = sums.fluidEnergy()
    time, step = 0.0, 0
    for k in range(spans):
        last = steps * (k + 1) // spans
        time, step, _ = sums.advance(time, step, math.inf, last, case.smoothingLength, case.cflNumber,
                                     case.maxTimeStep, case.densityFilterInterval)
    assert step == steps
    return sums, start, state


@pytest.mark.parametrize('tag', RUNS)
def test_the_device_budget_follows_the_references_and_closes(tag):
    r, case = budgetCase(tag)
    sums, start, _ = run(case, int(r['steps']))
    budget, end = sums.energySums(), sums.fluidEnergy()
    expected = r['budget'][:14]
    scale = np.abs(r['budget']).sum()
    # the fluid's energy is the reference's at the start and, to the run's own drift, at the end
    assert np.allclose(start, r['startEnergy'], rtol=1e-6, atol=1e-9 * scale)
    assert np.allclose(end, r['endEnergy'], rtol=0.0, atol=1e-3 * scale)
    for k, name in enumerate(energyTerms):
        assert budget[k] == pytest.approx(expected[k], abs=1e-3 * scale), name
    assert budget.sum() == pytest.approx((end - start).sum(), abs=1e-5 * np.abs(budget).sum())
    if tag in ('channel', 'published', 'hybrid'):
        assert budget[energyTerms.index('viscosityFluid')] <= 0.0


def test_the_budget_closes_across_advance_calls():
    # tests/testSphEnergy.py:189-203: the totals run from the push through every call
    r, case = budgetCase('channel')
    sums, start, _ = run(case, int(r['steps']), spans=3)
    budget, end = sums.energySums(), sums.fluidEnergy()
    assert budget.sum() == pytest.approx((end - start).sum(), abs=1e-5 * np.abs(budget).sum())
    whole, _, _ = run(case, int(r['steps']))
    assert np.array_equal(budget, whole.energySums())


def test_the_budget_leaves_the_device_step_alone():
    # tests/testSphEnergy.py:243-253: the tracked run is the plain run, bit for bit
    for tag in ('channel', 'shifted', 'filtered'):
        r, tracked = budgetCase(tag, track=True)
        _, plain = budgetCase(tag, track=False)
        a, _, _ = run(tracked, int(r['steps']))
        b, _, _ = run(plain, int(r['steps']))
        sa, sb = tracked.state.copy(), plain.state.copy()
        a.pull(sa)
        b.pull(sb)
        for name in ('positions', 'velocities', 'densities'):
            assert np.array_equal(getattr(sa, name), getattr(sb, name)), (tag, name)


def test_the_budget_is_off_until_asked_and_restarts_at_the_push():
    r, case = budgetCase('channel', track=False)
    sums, _, state = run(case, 5)
    with pytest.raises(ValueError):
        sums.energySums()
    sums.setEnergyBudget(True)
    sums.push(case.state.copy())
    assert not np.any(sums.energySums())


def test_a_split_keeps_the_totals_and_its_change_is_the_refinement():
    # src/pysurf/sphSolver.py:2000-2060 (refine): the refinement term is the split's change of K + P + E_C;
    # with it the budget closes over a run that splits its crest between device calls
    r, case = budgetCase('channel')
    sums, start, state = run(case, 10)
    before = sums.fluidEnergy()
    kept = sums.energySums()
    pulled = case.state.copy()
    sums.pull(pulled)
    crest = np.asarray(pulled.isFluid) & (pulled.positions[:, 1] > 0.8)
    assert sums.split(crest, case.referenceDensity) > 0
    assert np.array_equal(sums.energySums(), kept)
    refinement = (sums.fluidEnergy() - before).sum()
    time, step, _ = sums.advance(0.0, 10, math.inf, 20, case.smoothingLength, case.cflNumber, case.maxTimeStep,
                                 case.densityFilterInterval)
    assert step == 20
    budget, end = sums.energySums(), sums.fluidEnergy()
    assert (budget.sum() + refinement) == pytest.approx((end - start).sum(), abs=1e-5 * np.abs(budget).sum())
