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
        # The format: arrays positions, speeds, then the caller's fields (one row a fluid particle) in
        # frameNNNNN.npz; an index entry {frame, time, step, count, file, scalars...}; the index
        # {"frames": [...]} rewritten whole, one-space indent, after every frame.
        count = int(np.shape(speeds)[0])
        extra = {name: np.asarray(values) for name, values in (fields or {}).items()}
        wrong = {name: len(values) for name, values in extra.items() if len(values) != count}
        if wrong:
            name, rows = next(iter(wrong.items()))
            raise ValueError(f"Field '{name}' has {rows} rows for {count} fluid particles.")
        number = len(self.frames)
        path = self.directory / _frameName(number)
        save = np.savez_compressed if self.compress else np.savez
        save(path, positions=positions, speeds=speeds, **extra)
        self.frames.append(_indexEntry(number, time, step, count, path.name, scalars))
        _writeIndex(self.directory, self.frames)
        return path


def _frameName(number: int) -> str:
    return f'frame{number:05d}.npz'


def _indexEntry(number: int, time: float, step, count: int, file: str, scalars: dict | None) -> dict:
    entry = dict(frame=number, time=float(time), step=step, count=count, file=file)
    for name, value in (scalars or {}).items():
        entry[name] = float(value)
    return entry


def _writeIndex(directory: Path, entries: list) -> None:
    (directory / INDEX).write_text(json.dumps({'frames': entries}, indent=1), encoding='utf-8')


def readIndex(directory) -> list[dict]:
    """A run's index: one entry a frame, in order."""
    with open(Path(directory) / INDEX, 'r', encoding='utf-8') as handle:
        return json.load(handle)['frames']


def readFrame(directory, frame: int) -> dict:
    """One frame's arrays: positions, speeds and the fields written with it."""
    entry = readIndex(directory)[frame]
    with np.load(Path(directory) / entry['file'], allow_pickle=False) as data:
        return {name: data[name] for name in data.files}
