"""The breaking tracker (pysurf_b200.breaking) against the reference's own measures.

tests/golden/breaking.npz holds the reference's freeSurfaceProfile, frontFaceLean, troughAhead,
waterlineX and a BreakingTracker fed a sequence of shapes (src/pysurf/waveBreaking.py, the 'cells'
face), computed by tests/golden/make_golden.py on synthetic fluid shapes over a 1:15 beach: still
water, a steep crest, lips leaning over the face, and the same jittered.
"""
import numpy as np
import pytest

from pysurf_b200 import breaking
from pysurf_b200.state import Profile

SHAPES = ['still', 'steep', 'lip1', 'lip3', 'still_jitter', 'steep_jitter', 'lip1_jitter', 'lip3_jitter']
SPACING = 1.0 / 16.0


@pytest.fixture(scope='module')
def data():
    from conftest import GOLDEN
    import os
    with np.load(os.path.join(GOLDEN, 'breaking.npz')) as f:
        return {k: f[k] for k in f.files}


@pytest.fixture(scope='module')
def bed(data):
    return Profile(data['bed/x'], data['bed/z'], 1.0)


@pytest.mark.parametrize('shape', SHAPES)
def test_the_measures_match_the_reference(data, bed, shape):
    points = data[f'{shape}/positions']
    centers, elevation = breaking.surfaceProfile(points, bed.startX, bed.endX, SPACING)
    assert np.array_equal(centers, data[f'{shape}/centers'])
    assert np.array_equal(elevation, data[f'{shape}/elevation'], equal_nan=True)
    crestX = float(centers[int(np.nanargmax(elevation))])
    assert breaking.faceLean(points, crestX, 1.0, SPACING, 1.0) == float(data[f'{shape}/lean'])
    assert breaking.troughAhead(centers, elevation, crestX, 2.0) == float(data[f'{shape}/trough'])
    assert breaking.waterlineX(points, bed, 2.0 * SPACING) == float(data[f'{shape}/waterline'])


def test_the_tracker_finds_the_reference_breaking_point(data, bed):
    tracker = breaking.BreakingTracker(bed, SPACING, faceReach=1.0, searchFromX=15.0)
    for k, name in enumerate(data['sequence']):
        tracker.update(0.1 * (k + 1), data[f'{name}/positions'])
    assert np.array_equal(tracker.crestX, data['tracker/crestX'])
    assert np.array_equal(tracker.crestHeight, data['tracker/crestHeight'])
    assert np.array_equal(tracker.lean, data['tracker/lean'])
    assert np.array_equal(tracker.waterline, data['tracker/waterline'], equal_nan=True)
    assert tracker.maxRunup == float(data['tracker/maxRunup'])
    point = tracker.breakingPoint
    assert point is not None and tracker.breakingFinal
    expected = data['tracker/point']
    got = np.array([point.time, point.lean, point.crestX, point.crestHeight, point.depth, point.troughHeight])
    assert np.array_equal(got, expected)


def test_a_lean_must_persist_three_updates(data, bed):
    tracker = breaking.BreakingTracker(bed, SPACING, faceReach=1.0, searchFromX=15.0)
    for k, name in enumerate(['lip1', 'lip1_jitter', 'steep', 'lip1', 'lip1_jitter']):
        tracker.update(0.1 * k, data[f'{name}/positions'])
    assert tracker.breakingPoint is None
    tracker.update(1.0, data['lip1/positions'])
    assert tracker.breakingPoint is not None and tracker.breakingPoint.time == pytest.approx(0.3)
