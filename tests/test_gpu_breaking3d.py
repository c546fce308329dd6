"""The 3D breaking tracker's section reads on the device, and a 3D run to the breaking point against the
float64 step, to 1% in time and crest.

The 3D facade reads each section's fluid -- the particles within sectionRows / 2 spacings of the
section's y -- in its (x, z) plane (BreakingWave3D._readSections, src/pysurf/BreakingWave3D.py:461-480).
The device takes a section's reads (column tops, face cells, the bed's sheet) over that band; they must
equal the host's reads of the pulled positions bit for bit.  The run to breaking is the 2D beach's start
extruded across a periodic y axis (cases.extrudedBeach: H/d 0.6 over a 1:15 beach, 8 ppd, 14 columns
across, deltaSph scheme at h = 3 dx), its middle section read every 0.01 sqrt(d / g), once on the B200
and once with the oracle's float64 step on the host.
"""
import math

import numpy as np
import pytest

from oracle import oracle
from pysurf_b200 import breaking, cases

pytestmark = pytest.mark.gpu


def pushed(case):
    sums = cases.pairSumsFor(case)
    state = case.state.copy()
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    return sums


@pytest.mark.parametrize('build', [lambda: cases.ridgeWave3D(6, length=12.0, width=3.0, crestX=4.0, ridgeX=7.0),
                                   lambda: cases.extrudedBeach(8)])
def test_the_device_reads_a_section_as_the_host_does(build):
    case = build()
    sums = pushed(case)
    width = float(case.info['tank'][1]) if 'tank' in case.info else float(case.info['width'])
    onDevice = breaking.sectionTrackers(case, sections=(0.5 * width, 0.3 * width))
    onHost = breaking.sectionTrackers(case, sections=(0.5 * width, 0.3 * width))
    time, step, dt = 0.0, 0, 0.0
    for target in np.linspace(0.05, 0.6, 6):
        time, step, dt = sums.advance(time, step, float(target), 1 << 40, case.smoothingLength, case.cflNumber,
                                      case.maxTimeStep, 0, dt)
        state = sums.pullState()
        fluid = state['positions'][state['isFluid']]
        for y in onDevice:
            onDevice[y].updateOnDevice(time, sums)
            onHost[y].update(time, onHost[y].sectionOf(fluid))
    for y in onDevice:
        a, b = onDevice[y], onHost[y]
        assert len(b.times) == 6 and np.isfinite(b.crestX).all()
        for name in ('crestX', 'crestHeight', 'lean', 'waterline'):
            assert np.array_equal(getattr(a, name), getattr(b, name), equal_nan=True), (y, name)


def oracleToBreaking(case, endTime: float):
    bed = case.boundary.bathymetry
    stepper = oracle.Stepper(3, case.kernelType, case.smoothingLength, case.referenceDensity, case.soundSpeed,
                             case.alpha, case.gravity, 0.0, 0.0, case.densityFloor, case.densityDiffusion,
                             case.diffusionDelta, True, False, True, True, case.cflNumber, case.maxTimeStep,
                             case.period, 0, ('bed', oracle.bedParams(bed.x, bed.z, 0.25 * case.spacing, False, 0.0,
                                                                      True, bed.startX, 0.0, bed.endX)))
    state = {k: np.array(getattr(case.state, k), copy=True)
             for k in ('positions', 'velocities', 'densities', 'masses', 'isFluid')}
    fluid = np.asarray(case.state.isFluid, dtype=bool)
    tracker = next(iter(breaking.sectionTrackers(case).values()))
    interval = 0.01 * math.sqrt(float(case.info['depth']) / 9.80665)
    nextTrack = interval
    while stepper.time < endTime and not tracker.breakingFinal:
        while stepper.time < nextTrack:
            stepper(state)
        tracker.update(stepper.time, tracker.sectionOf(state['positions'][fluid]))
        nextTrack += interval
    return tracker


def test_the_3d_device_breaks_where_the_float64_step_breaks():
    case = cases.extrudedBeach(8)
    device, time, steps = breaking.runToBreaking(case, pushed(case), endTime=4.0)
    reference = oracleToBreaking(case, 4.0)
    a, b = device.breakingPoint, reference.breakingPoint
    assert a is not None and b is not None
    print(f'\nextruded beach, {case.fluidCount} fluid particles: device breaks at t = {a.time:.4f} s, crest '
          f'{a.crestX:.4f} m; float64 at t = {b.time:.4f} s, crest {b.crestX:.4f} m')
    assert abs(a.time - b.time) <= 0.01 * b.time
    assert abs(a.crestX - b.crestX) <= 0.01 * b.crestX
    assert abs(a.crestHeight - b.crestHeight) <= 0.05 * b.crestHeight
