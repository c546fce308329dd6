"""Frames and checkpoints from the device state.

A frame written from the device (``FrameWriter.writeDevice``, ``sph_frame``) holds the bits the
reference's FrameWriter writes from the pulled state; a run taken up from a checkpoint of its device
state continues bit for bit (tests/testBreakingWave3D.py:266-296 asks the same of the reference's).
"""
import math

import numpy as np
import pytest

from pysurf_b200 import cases, checkpoint, frames
from test_frames_host import GOLDEN, goldenState

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('tag', ['frames2d', 'frames3d'])
def test_a_device_frame_is_the_references(tag, tmp_path):
    from pysurf_b200.sphGpu import PairSums
    p = goldenState(tag)
    x = p.positions
    sums = PairSums(x.shape[1], float(p.lengths.max()), x.min(axis=0), x.max(axis=0), device='cuda:0')
    sums.push(p)
    writer = frames.FrameWriter(tmp_path)
    count = int(np.sum(p.isFluid))
    writer.writeDevice(0.25, sums, step=7, fields={'ids': np.arange(count)}, scalars={'energy': 1.5})
    writer.writeDevice(0.5, sums, step=9)
    assert (tmp_path / 'frames.json').read_text(encoding='utf-8') == str(GOLDEN[f'{tag}/index'])
    for frame in (0, 1):
        got = frames.readFrame(tmp_path, frame)
        for name in ('positions', 'speeds'):
            expected = GOLDEN[f'{tag}/frame{frame}_{name}']
            assert got[name].dtype == expected.dtype and np.array_equal(got[name], expected), name


def test_a_checkpoint_continues_the_run_as_if_it_had_not_stopped(tmp_path):
    # a split beach (masses and lengths of the zone in the checkpoint), 15 steps, checkpoint, 15 more;
    # taken up from the checkpoint in a fresh PairSums, the 15 more steps give the same bits
    case = cases.solitaryBeach(particlesPerDepth=8)
    state = case.state.copy()
    crest = state.isFluid & (state.positions[:, 0] > 8.0) & (state.positions[:, 0] < 12.0)
    sums = cases.pairSumsFor(case)
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    sums.split(crest, case.referenceDensity, 0.5)
    shortest = float(sums.pullState()['lengths'].min())
    time, step, dt = sums.advance(0.0, 0, math.inf, 15, shortest, case.cflNumber, case.maxTimeStep)
    path = tmp_path / 'run.pkl'
    checkpoint.saveCheckpoint(path, sums, {'time': time, 'step': step, 'timeStep': dt}, {'ppd': 8}, mergedGroups=0)
    assert not (tmp_path / 'run.pkl.partial').exists()
    time, step, dt = sums.advance(time, step, math.inf, 30, shortest, case.cflNumber, case.maxTimeStep, 0, dt)
    unbroken = sums.pullState()

    resumed = cases.pairSumsFor(case)
    clock = checkpoint.restoreCheckpoint(path, resumed, case.boundary, {'ppd': 8})
    assert clock['step'] == 15
    t2, s2, dt2 = resumed.advance(clock['time'], clock['step'], math.inf, 30, shortest, case.cflNumber,
                                  case.maxTimeStep, 0, clock['timeStep'])
    assert (t2, s2, dt2) == (time, step, dt)
    again = resumed.pullState()
    for name in ('positions', 'velocities', 'densities', 'masses', 'lengths', 'isFluid'):
        assert np.array_equal(again[name], unbroken[name]), name
    saved = checkpoint.loadCheckpoint(path)
    assert tuple(saved['particles']) == checkpoint.PARTICLE_FIELDS and saved['mergedGroups'] == 0
