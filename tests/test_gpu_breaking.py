"""A full run to the breaking point: the device against the float64 step, to 1% in time and crest.

The 16-ppd solitary wave (H/d 0.45, 1:15 beach, deltaSph scheme) runs from its start until the
breaking tracker (the reference's 'cells' face measure, pysurf_b200.breaking) records the breaking
point, once on the B200 and once with the oracle's float64 step on the host, the tracker reading
both every 0.01 sqrt(d / g).  Breaking time and crest position must agree within 1%.
"""
import math
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from pysurf_b200 import breaking, cases  # noqa: E402

pytestmark = pytest.mark.gpu


def oracleToBreaking(case, endTime: float):
    import bench
    stepper = bench.oracleStepper(case)
    state = {k: np.array(getattr(case.state, k), copy=True)
             for k in ('positions', 'velocities', 'densities', 'masses', 'isFluid')}
    fluid = np.asarray(case.state.isFluid, dtype=bool)
    tracker = breaking.trackerFor(case)
    interval = 0.01 * math.sqrt(float(case.info['depth']) / 9.80665)
    nextTrack = interval
    while stepper.time < endTime and not tracker.breakingFinal:
        while stepper.time < nextTrack:
            stepper(state)
        tracker.update(stepper.time, state['positions'][fluid])
        nextTrack += interval
    return tracker


def test_the_device_breaks_where_the_float64_step_breaks():
    case = cases.solitaryBeach(16)
    sums = cases.pairSumsFor(case)
    state = case.state.copy()
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    device, time, steps = breaking.runToBreaking(case, sums, endTime=6.0)
    reference = oracleToBreaking(case, 6.0)
    a, b = device.breakingPoint, reference.breakingPoint
    assert a is not None and b is not None
    assert abs(a.time - b.time) <= 0.01 * b.time
    assert abs(a.crestX - b.crestX) <= 0.01 * b.crestX
    assert abs(a.crestHeight - b.crestHeight) <= 0.05 * b.crestHeight


def test_the_device_reads_the_wave_as_the_host_does():
    # the device's reductions give the tracker what pulled positions give it, to the last bit
    case = cases.solitaryBeach(16)
    sums = cases.pairSumsFor(case)
    state = case.state.copy()
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    fluid = np.asarray(case.state.isFluid, dtype=bool)
    onDevice, onHost = breaking.trackerFor(case), breaking.trackerFor(case)
    time, step, dt = 0.0, 0, 0.0
    for target in np.linspace(0.2, 4.0, 12):
        time, step, dt = sums.advance(time, step, float(target), 1 << 40, case.smoothingLength, case.cflNumber,
                                      case.maxTimeStep, 0, dt)
        onDevice.updateOnDevice(time, sums)
        onHost.update(time, sums.pullPositions()[fluid])
    for name in ('crestX', 'crestHeight', 'lean', 'waterline'):
        assert np.array_equal(getattr(onDevice, name), getattr(onHost, name), equal_nan=True), name
    assert onDevice.maxRunup == onHost.maxRunup or (np.isnan(onDevice.maxRunup) and np.isnan(onHost.maxRunup))
    assert (onDevice.breakingPoint is None) == (onHost.breakingPoint is None)
    if onHost.breakingPoint is not None:
        assert onDevice.breakingPoint == onHost.breakingPoint
