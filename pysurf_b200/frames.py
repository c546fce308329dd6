"""A run's frames on disk, written from the device state (src/pysurf/sphFrames.py).

The reference streams an SPH run to a directory, one ``.npz`` file a frame and an index,
``frames.json``, rewritten after every frame so that a run cut short stays readable.  A frame holds
the fluid particles' float32 positions and float32 speeds, with any per-particle fields and scalars
the caller adds.  This module writes the same files, so the reference's ``readIndex`` and
``readFrame`` read them, and its own readers read the reference's:

    FrameWriter.write          a frame from a particle state on the host, as the reference writes it
    FrameWriter.writeDevice    the same frame from a ``PairSums``' device state: the device rounds
                               positions and speeds to float32 itself (``sph_frame``), so 17 bytes a
                               particle cross the bus instead of a float64 pull's 48
    readIndex, readFrame       a run's index and one frame's arrays
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

INDEX = 'frames.json'


class FrameWriter:
    """One ``frameNNNNN.npz`` a frame in `directory` (created if missing), indexed in ``frames.json``;
    `compress` writes compressed files (src/pysurf/sphFrames.py:38-100)."""

    def __init__(self, directory, compress: bool = False) -> None:
        self.directory = Path(directory)
        self.directory.mkdir(parents=True, exist_ok=True)
        self.compress = bool(compress)
        self.frames: list[dict] = []

    def write(self, time: float, particles, step: int | None = None, fields: dict | None = None,
              scalars: dict | None = None) -> Path:
        """The fluid's state at `time` from host arrays (positions, velocities, isFluid)."""
        fluid = np.asarray(particles.isFluid, dtype=bool)
        positions = np.asarray(particles.positions)[fluid].astype(np.float32)
        speeds = np.linalg.norm(np.asarray(particles.velocities)[fluid], axis=1).astype(np.float32)
        return self._store(time, positions, speeds, step, fields, scalars)

    def writeDevice(self, time: float, sums, step: int | None = None, fields: dict | None = None,
                    scalars: dict | None = None) -> Path:
        """The fluid's state at `time` from a PairSums' device state, the same bits as `write` of its pull."""
        positions, speeds = sums.frame()
        return self._store(time, positions, speeds, step, fields, scalars)

    def _store(self, time, positions, speeds, step, fields, scalars) -> Path:
        arrays = {'positions': positions, 'speeds': speeds}
        count = len(speeds)
        for name, values in (fields or {}).items():
            values = np.asarray(values)
            if len(values) != count:
                raise ValueError(f"Field '{name}' has {len(values)} rows for {count} fluid particles.")
            arrays[name] = values
        number = len(self.frames)
        path = self.directory / f'frame{number:05d}.npz'
        (np.savez_compressed if self.compress else np.savez)(path, **arrays)
        entry = {'frame': number, 'time': float(time), 'step': step, 'count': count, 'file': path.name}
        entry.update({name: float(value) for name, value in (scalars or {}).items()})
        self.frames.append(entry)
        with open(self.directory / INDEX, 'w', encoding='utf-8') as handle:
            json.dump({'frames': self.frames}, handle, indent=1)
        return path


def readIndex(directory) -> list[dict]:
    """A run's index: one entry a frame, in order."""
    with open(Path(directory) / INDEX, 'r', encoding='utf-8') as handle:
        return json.load(handle)['frames']


def readFrame(directory, frame: int) -> dict:
    """One frame's arrays: positions, speeds and the fields written with it."""
    entry = readIndex(directory)[frame]
    with np.load(Path(directory) / entry['file'], allow_pickle=False) as data:
        return {name: data[name] for name in data.files}
