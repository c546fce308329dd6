"""Failure detection on the device, made on the host: the step raises flags in its control block
instead of faulting, the device loop stops at the step that raised them, and the host reads them
as status codes.  Nothing here faults or waits on the GPU: a NaN density in the pushed state makes
the state non-finite within one step; a zero CFL number, which could only collapse the time step,
is refused on the host.  After either, the same handle takes a clean state and steps on."""
import math

import numpy as np
import pytest

from pysurf_b200 import _lib, cases

pytestmark = pytest.mark.gpu


def sloshing():
    case = cases.sloshingTank()
    sums = cases.pairSumsFor(case)
    return case, sums


def steps(sums, case, count, cfl=None):
    return sums.advance(0.0, 0, math.inf, count, case.smoothingLength, case.cflNumber if cfl is None else cfl,
                        case.maxTimeStep, case.densityFilterInterval)


def test_a_non_finite_state_stops_the_device_loop_and_the_handle_steps_on():
    case, sums = sloshing()
    bad = case.state.copy()
    bad.densities[np.flatnonzero(bad.isFluid)[0]] = np.nan
    sums.push(bad)
    sums.setBoundary(case.boundary, bad)
    with pytest.raises(_lib.SphError) as failure:
        steps(sums, case, 10)
    assert failure.value.status == _lib.SPH_ERR_NONFINITE
    # the same handle, a clean state: the run is the one a fresh handle makes
    good = case.state.copy()
    sums.push(good)
    sums.setBoundary(case.boundary, good)
    assert steps(sums, case, 10)[1] == 10
    sums.pull(good)
    fresh, other = cases.pairSumsFor(case), case.state.copy()
    fresh.push(other)
    fresh.setBoundary(case.boundary, other)
    steps(fresh, case, 10)
    fresh.pull(other)
    assert np.array_equal(good.positions, other.positions)
    assert np.array_equal(good.densities, other.densities)


def test_a_step_that_could_only_collapse_is_refused_before_it_runs():
    # a CFL number of zero would make every time step zero; the host refuses it, and the handle steps on
    case, sums = sloshing()
    state = case.state.copy()
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    with pytest.raises(ValueError):
        steps(sums, case, 5, cfl=0.0)
    assert steps(sums, case, 5)[1] == 5


def test_bad_arguments_are_refused_before_any_launch():
    case, sums = sloshing()
    with pytest.raises(ValueError):
        sums.setPhysics(-1.0, case.soundSpeed, case.alpha, 0.0, case.gravity, 0.0, 0.0)
    with pytest.raises(ValueError):
        sums.split(np.ones(3, dtype=bool), case.referenceDensity)
