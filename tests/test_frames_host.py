"""Frame files and checkpoints in the reference's layouts (src/pysurf/sphFrames.py;
src/pysurf/BreakingWave3D.py:204, 785-858), against files the reference wrote
(tests/golden/frames.npz, made by tests/golden/make_golden.py)."""
import pickle

import numpy as np
import pytest

from pysurf_b200 import checkpoint, frames
from pysurf_b200.state import ParticleState

GOLDEN = np.load('tests/golden/frames.npz')


def goldenState(tag):
    n, dim = GOLDEN[f'{tag}/state_positions'].shape
    return ParticleState(GOLDEN[f'{tag}/state_positions'], GOLDEN[f'{tag}/state_velocities'], np.zeros((n, dim)),
                         np.full(n, 1000.0), np.zeros(n), GOLDEN[f'{tag}/state_masses'],
                         GOLDEN[f'{tag}/state_isFluid'], GOLDEN[f'{tag}/state_lengths'])


@pytest.mark.parametrize('tag', ['frames2d', 'frames3d'])
def test_frames_are_the_references_file_for_file(tag, tmp_path):
    p = goldenState(tag)
    writer = frames.FrameWriter(tmp_path)
    count = int(np.sum(p.isFluid))
    writer.write(0.25, p, step=7, fields={'ids': np.arange(count)}, scalars={'energy': 1.5})
    writer.write(0.5, p, step=9)
    assert (tmp_path / 'frames.json').read_text(encoding='utf-8') == str(GOLDEN[f'{tag}/index'])
    for frame in (0, 1):
        got = frames.readFrame(tmp_path, frame)
        expected = {k.split('_', 1)[1]: GOLDEN[k] for k in GOLDEN.files if k.startswith(f'{tag}/frame{frame}_')}
        assert set(got) == set(expected)
        for name, values in expected.items():
            assert got[name].dtype == values.dtype and np.array_equal(got[name], values), name


def test_a_field_of_the_wrong_length_is_refused(tmp_path):
    with pytest.raises(ValueError):
        frames.FrameWriter(tmp_path).write(0.0, goldenState('frames2d'), fields={'bad': np.zeros(3)})


def test_the_checkpoint_layout_is_the_references():
    assert checkpoint.FORMAT == str(GOLDEN['checkpoint/format'])
    assert checkpoint.PARTICLE_FIELDS == tuple(GOLDEN['checkpoint/particleFields'])


def test_a_checkpoint_of_another_format_or_run_is_refused(tmp_path):
    other = tmp_path / 'other.pkl'
    other.write_bytes(pickle.dumps({'format': 'something else'}))
    with pytest.raises(ValueError):
        checkpoint.loadCheckpoint(other)
    mine = tmp_path / 'mine.pkl'
    mine.write_bytes(pickle.dumps({'format': checkpoint.FORMAT, 'settings': {'ppd': 8}}))
    assert checkpoint.loadCheckpoint(mine, {'ppd': 8})['settings'] == {'ppd': 8}
    with pytest.raises(ValueError):
        checkpoint.loadCheckpoint(mine, {'ppd': 16})
