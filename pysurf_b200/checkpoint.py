"""Checkpoints of a run's device state in the reference's layout (src/pysurf/BreakingWave3D.py:785-858).

The reference's 3D facade saves a run between calls to ``run`` as a pickle: a format tag, the
settings the run must match, the particles as the fields of its ``ParticleSystem`` (densities,
pressures and a split zone's masses and lengths included), the solver's clock and the facade's
own records.  The file is written to a partial file first, which then replaces any earlier
checkpoint, so a crash while writing leaves the earlier one whole.  Here the particles come from
the device state of a ``PairSums``, and a restore pushes them back, so a run taken up from a
checkpoint continues as if it had not stopped, bit for bit (the device's sums run in a fixed order).

    FORMAT, PARTICLE_FIELDS     the reference's format tag and ParticleSystem field order
    deviceParticles             the particle fields from a PairSums' device state
    saveCheckpoint              the pickle, written through a partial file
    loadCheckpoint              read one back, checking its format and settings
    restoreCheckpoint           push a checkpoint's particles into a PairSums; returns its clock

Load only checkpoints written by this code or the reference: unpickling runs code.
"""
from __future__ import annotations

import os
import pickle
from pathlib import Path

import numpy as np

FORMAT = 'pysurf.BreakingWave3D checkpoint 1'
PARTICLE_FIELDS = ('positions', 'velocities', 'accelerations', 'densities', 'pressures', 'masses', 'isFluid', 'lengths')


def deviceParticles(sums) -> dict:
    """The device state as the reference's ParticleSystem fields, in their order; lengths stay None
    while every particle has the PairSums' smoothing length, as the reference keeps them until a split."""
    state = sums.pullState()
    lengths = state['lengths']
    uniform = len(lengths) == 0 or bool(np.all(lengths == sums.smoothingLength))
    fields = {'positions': state['positions'], 'velocities': state['velocities'],
              'accelerations': state['accelerations'], 'densities': state['densities'],
              'pressures': state['pressures'], 'masses': state['masses'],
              'isFluid': np.asarray(state['isFluid'], dtype=bool), 'lengths': None if uniform else lengths}
    return {name: fields[name] for name in PARTICLE_FIELDS}


def saveCheckpoint(path, sums, clock: dict, settings: dict | None = None, **records) -> Path:
    """Write the device state with `clock` ({'time', 'step', 'timeStep'}), the `settings` a restore must
    match and any further `records` (the facade's trackers, tallies, wall clock) to `path`."""
    path = Path(path)
    state = {'format': FORMAT, 'settings': settings, 'particles': deviceParticles(sums),
             'clock': {'time': float(clock['time']), 'step': int(clock['step']),
                       'timeStep': float(clock['timeStep'])}}
    state.update(records)
    partial = path.with_name(path.name + '.partial')
    with open(partial, 'wb') as handle:
        pickle.dump(state, handle, protocol=5)
    os.replace(partial, path)
    return path


def loadCheckpoint(path, settings: dict | None = None) -> dict:
    """A checkpoint's contents; ValueError when it is not one of this format, or when `settings` are
    given and the run that wrote it had others."""
    with open(path, 'rb') as handle:
        state = pickle.load(handle)
    if not isinstance(state, dict) or state.get('format') != FORMAT:
        raise ValueError('The file is not a BreakingWave3D checkpoint of this format.')
    if settings is not None and state.get('settings') != settings:
        raise ValueError('A run with other settings wrote the checkpoint.')
    return state


def restoreCheckpoint(path, sums, boundary=None, settings: dict | None = None) -> dict:
    """Push a checkpoint's particles into `sums` (and set `boundary` on them); returns its clock."""
    from pysurf_b200.state import ParticleState
    state = loadCheckpoint(path, settings)
    p = state['particles']
    particles = ParticleState(np.array(p['positions']), np.array(p['velocities']), np.array(p['accelerations']),
                              np.array(p['densities']), np.array(p['pressures']), np.array(p['masses']),
                              np.array(p['isFluid'], dtype=bool),
                              None if p['lengths'] is None else np.array(p['lengths']))
    sums.push(particles)
    if boundary is not None:
        sums.setBoundary(boundary, particles)
    return dict(state['clock'])
