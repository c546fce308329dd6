"""Where a wave breaks: the breaking tracker of the reference's 2D facade, and its 3D sections.

The reference reads the wave from the fluid's positions every 0.01 sqrt(d / g) of simulated time
(src/pysurf/BreakingWave.py:885-912) with `BreakingTracker` (src/pysurf/waveBreaking.py:709-906).
This module restates its 'cells' face measure, the one its first-order (lattice) start uses:

    surfaceProfile  the free surface column by column: the highest fluid particle of each column one
                    spacing wide, plus half a spacing (waveBreaking.py:129-162)
    troughAhead     the lowest surface shoreward of the crest, after a three-column running median
                    (waveBreaking.py:164-204)
    faceLean        how far the crest's shoreward face leans past vertical, read in cells one spacing
                    square above still water (waveBreaking.py:559-634)
    waterlineX      the landward tip of the water sheet on the bed (waveBreaking.py:636-656)
    BreakingTracker the crest's history and the breaking point: the first of `persistence`
                    consecutive updates with the face leaning a spacing or more, with the crest past
                    `searchFromX` (waveBreaking.py:709-906, the 'cells' branch)

In 3D the reference reads sections across the tank (BreakingWave3D._readSections,
src/pysurf/BreakingWave3D.py:461-480): each section's tracker takes the fluid within half its
width (sectionRows / 2 spacings) of its y, in the (x, z) plane, over the bed's profile along x at
that y.  The facade reads them with the 'contour' face measure, which contours a smoothed fluid
fraction with the third-party contourpy (not in this image); these sections read the 'cells'
measure, the same lean, trough and waterline as the 2D tracker, over each section's fluid.

`runToBreaking` steps a `PairSums` on the device to the breaking point.  At each tracker update the
device takes the reductions an update needs (each column's highest particle, the face window's
cells, the x of the bed's water sheet: sph_surface_tops, sph_face_cells, sph_bed_sheet, and in 3D
the sph_section_* reads over a section's band) with the float64 arithmetic of the host's measures,
and only those come back; `updateOnDevice` then reads them as `update` reads pulled positions, to
the same values.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


def surfaceProfile(positions: np.ndarray, x0: float, x1: float, width: float) -> tuple[np.ndarray, np.ndarray]:
    """Column centres over [x0, x1) and each column's surface: its highest particle plus half a
    column; NaN where a column holds no particle."""
    count = max(1, int(math.ceil((x1 - x0) / width)))
    centers = x0 + (np.arange(count) + 0.5) * width
    column = np.floor((positions[:, 0] - x0) / width).astype(np.int64)
    inside = (column >= 0) & (column < count)
    top = np.full(count, -np.inf)
    if inside.any():
        np.maximum.at(top, column[inside], positions[inside, 1])
    return centers, np.where(np.isfinite(top), top + 0.5 * width, np.nan)


def troughAhead(centers: np.ndarray, elevation: np.ndarray, crestX: float, reach: float = np.inf) -> float:
    """The least surface among the wet columns from the crest shoreward, up to the first dry column
    or `reach` past the crest, after a running median over three columns with the ends reflected;
    NaN when the first column ahead is dry."""
    ahead = np.flatnonzero((centers > crestX) & (centers <= crestX + reach))
    levels = np.asarray(elevation, dtype=float)[ahead]
    dry = np.flatnonzero(~np.isfinite(levels))
    if dry.size:
        levels = levels[:dry[0]]
    if levels.size == 0:
        return float('nan')
    if levels.size < 3:
        return float(levels.max())
    padded = np.concatenate([levels[1:2], levels, levels[-2:-1]])
    windows = np.stack([padded[:-2], padded[1:-1], padded[2:]])
    return float(np.median(windows, axis=0).min())


def faceLean(positions: np.ndarray, crestX: float, stillWaterLevel: float, spacing: float, reach: float,
             shoreLimit: float = np.inf) -> float:
    """How far the crest's shoreward face leans forward of vertical [m]: negative sloping back, zero
    vertical, positive curling over; -inf when fewer than two bands show a face.

    The window runs from half a spacing behind the crest to `reach` ahead of it (or `shoreLimit`),
    above still water plus half a spacing, in cells one spacing square.  A particle marks the four
    cells its own square (a spacing across, centred on it) overlaps.  In each band the face is the
    shoreward end of the run of marked cells that starts in one of the first two columns; bands whose
    run reaches the window's end are left out.  The lean is the most any band's face stands
    shoreward of the face of a band below it."""
    start = crestX - 0.5 * spacing
    end = min(crestX + reach, shoreLimit)
    base = stillWaterLevel + 0.5 * spacing
    x, z = positions[:, 0], positions[:, 1]
    near = (x >= start - 0.5 * spacing) & (x < end + 0.5 * spacing) & (z > base - 0.5 * spacing)
    if not near.any():
        return -np.inf
    column0 = np.floor((x[near] - 0.5 * spacing - start) / spacing).astype(np.int64)
    band0 = np.floor((z[near] - 0.5 * spacing - base) / spacing).astype(np.int64)
    columns = max(1, int(math.ceil((end - start) / spacing)))
    marked = np.zeros((int(band0.max()) + 2, columns), dtype=bool)
    for dc in (0, 1):
        for db in (0, 1):
            c, b = column0 + dc, band0 + db
            keep = (c >= 0) & (c < columns) & (b >= 0)
            marked[b[keep], c[keep]] = True
    return leanOfCells(marked, start, spacing)


def leanOfCells(marked: np.ndarray, start: float, spacing: float) -> float:
    """The lean from the window's marked cells (bands bottom up, columns from `start`)."""
    faces = []
    for band in marked:
        first = np.flatnonzero(band[:2])
        if first.size == 0:
            continue
        run = band[first[0]:]
        gaps = np.flatnonzero(~run)
        if gaps.size == 0:
            continue
        faces.append(start + (first[0] + gaps[0]) * spacing)
    if len(faces) < 2:
        return -np.inf
    faces = np.asarray(faces)
    below = np.minimum.accumulate(faces)
    return float((faces[1:] - below[:-1]).max())


def waterlineX(positions: np.ndarray, bed, wetHeight: float, minimumParticles: int = 3) -> float:
    """The landward tip of the water on the bed: the `minimumParticles`-th most landward particle
    within `wetHeight` of the bed (so a lone droplet ahead of the sheet does not set it); NaN with
    fewer."""
    onBed = positions[positions[:, 1] - bed.elevation(positions[:, 0]) < wetHeight]
    if len(onBed) < minimumParticles:
        return float('nan')
    return float(np.partition(onBed[:, 0], len(onBed) - minimumParticles)[len(onBed) - minimumParticles])


@dataclass
class BreakingPoint:
    """The update the breaking point was read at: time, face lean, crest position and height above
    still water (Hb), still water depth under the crest (hb), and the trough ahead."""
    time: float
    lean: float
    crestX: float
    crestHeight: float
    depth: float
    faceX: float = float('nan')
    faceDepth: float = float('nan')
    troughHeight: float = float('nan')

    @property
    def breakingIndex(self) -> float:
        """Hb / hb."""
        return self.crestHeight / self.depth if self.depth > 0.0 else float('inf')

    @property
    def waveHeight(self) -> float:
        """Crest elevation less the trough's."""
        return self.crestHeight - self.troughHeight


@dataclass
class BreakingTracker:
    """The crest's history and the breaking point of a wave on a bed profile (the 'cells' measure):
    the first of `persistence` consecutive updates whose face leans at least `leanThreshold`
    spacings (less half a spacing, so rounding does not decide a tie), with the crest past
    `searchFromX`."""
    bed: object
    spacing: float
    leanThreshold: float = 1.0
    faceReach: float = 1.0
    searchFromX: float = -np.inf
    persistence: int = 3
    section: tuple | None = None    # 3D: (y, half width), the band across the tank this tracker reads
    times: list = field(default_factory=list)
    crestX: list = field(default_factory=list)
    crestHeight: list = field(default_factory=list)
    lean: list = field(default_factory=list)
    waterline: list = field(default_factory=list)
    breakingPoint: BreakingPoint | None = None
    maxRunup: float = float('nan')
    _candidate: BreakingPoint | None = field(default=None, repr=False)
    _streak: int = field(default=0, repr=False)

    @property
    def breakingFinal(self) -> bool:
        return self.breakingPoint is not None

    def sectionOf(self, positions: np.ndarray) -> np.ndarray:
        """This section's fluid in its (x, z) plane from the whole fluid's positions (N, 3)
        (src/pysurf/BreakingWave3D.py:461-480); 2D positions as they are."""
        if self.section is None:
            return positions
        y, half = self.section
        return positions[np.abs(positions[:, 1] - y) < half][:, [0, 2]]

    def update(self, time: float, positions: np.ndarray) -> None:
        """Read the wave from the fluid's positions (N, 2) at `time` (a section's: see `sectionOf`)."""
        bed, s = self.bed, self.spacing
        centers, elevation = surfaceProfile(positions, bed.startX, bed.endX, s)
        crestX = float(centers[int(np.nanargmax(elevation))])
        lean = faceLean(positions, crestX, bed.stillWaterLevel, s, self.faceReach)
        self.record(time, centers, elevation, lean, waterlineX(positions, bed, 2.0 * s))

    def updateOnDevice(self, time: float, sums) -> None:
        """The same reading from the state a `PairSums` holds, its reductions taken on the device
        (column tops, face cells, the bed's sheet): a few kilobytes come back instead of the positions."""
        bed, s = self.bed, self.spacing
        swl = bed.stillWaterLevel
        count = max(1, int(math.ceil((bed.endX - bed.startX) / s)))
        centers = bed.startX + (np.arange(count) + 0.5) * s
        band = self.section
        tops = sums.surfaceTops(bed.startX, s, count, section=band)
        elevation = np.where(np.isfinite(tops), tops + 0.5 * s, np.nan)
        crestX = float(centers[int(np.nanargmax(elevation))])
        # faceLean's window, its cells marked on the device; the bands reach the highest particle
        start, end, base, half = crestX - 0.5 * s, crestX + self.faceReach, swl + 0.5 * s, 0.5 * s
        columns = max(1, int(math.ceil((end - start) / s)))
        highest = float(np.max(tops[np.isfinite(tops)])) if np.isfinite(tops).any() else base
        bands = max(1, int(math.floor((highest - half - base) / s)) + 2)
        marked = sums.faceCells(start - half, end + half, base - half, half, start, base, s, columns, bands,
                                section=band)
        lean = leanOfCells(marked, start, s) if marked.any() else -np.inf
        sheet = sums.bedSheet(bed.x, bed.z, 2.0 * s, section=band)
        tip = float(np.partition(sheet, sheet.size - 3)[sheet.size - 3]) if sheet.size >= 3 else float('nan')
        self.record(time, centers, elevation, lean, tip)

    def record(self, time: float, centers: np.ndarray, elevation: np.ndarray, lean: float, tip: float) -> None:
        """Record an update from its reading: the surface profile, the face lean, the waterline."""
        bed, s = self.bed, self.spacing
        swl = bed.stillWaterLevel
        top = int(np.nanargmax(elevation))
        crestX, crestHeight = float(centers[top]), float(elevation[top] - swl)
        steep = lean > (self.leanThreshold - 0.5) * s
        trough = troughAhead(centers, elevation, crestX, 2.0 * self.faceReach) - swl
        if np.isfinite(tip):
            runup = float(bed.elevation(tip) - swl)
            self.maxRunup = runup if not np.isfinite(self.maxRunup) else max(self.maxRunup, runup)
        self.times.append(time)
        self.crestX.append(crestX)
        self.crestHeight.append(crestHeight)
        self.lean.append(lean)
        self.waterline.append(tip)
        if self.breakingPoint is not None:
            return
        if crestX >= self.searchFromX and steep:
            if self._streak == 0:
                self._candidate = BreakingPoint(time, lean, crestX, crestHeight, float(bed.depth(crestX)),
                                                troughHeight=trough)
            self._streak += 1
            if self._streak >= self.persistence:
                self.breakingPoint = self._candidate
        else:
            self._streak, self._candidate = 0, None


def trackerFor(case) -> BreakingTracker:
    """The facade's tracker for a beach case: face reach one depth, breaking looked for from the
    toe on (src/pysurf/BreakingWave.py:763-765)."""
    info = case.info
    return BreakingTracker(case.boundary.bathymetry, case.spacing, faceReach=float(info['depth']),
                           searchFromX=float(info['toeX']))


def sectionTrackers(case, sections=None, sectionRows: int = 2) -> dict:
    """The 3D facade's trackers, one a section (src/pysurf/BreakingWave3D.py:356-400, 690-694): the
    tank's middle line by default, each reading the fluid within sectionRows / 2 spacings of its y
    over the bed's profile along x there (cases.ridgeSection), face reach one depth, breaking looked
    for from the wave's start on; the 'cells' face measure (see the module's notes)."""
    from pysurf_b200 import cases
    info, s = case.info, case.spacing
    ridge = type(case.boundary).__name__ == 'HeightFieldBoundary'
    width = float(info['tank'][1]) if ridge else float(info['width'])
    ys = tuple(float(y) for y in (sections if sections is not None else (0.5 * width,)))
    half = 0.5 * sectionRows * s

    def profile(y):
        # a height field's section; an extruded beach's profile is the same at every y
        return cases.ridgeSection(case, y) if ridge else case.boundary.bathymetry

    # the 3D facade looks for breaking from the wave's start, the 2D one from the beach's toe
    searchFromX = float(info['crestX']) if ridge else float(info['toeX'])
    return {y: BreakingTracker(profile(y), s, faceReach=float(info['depth']), searchFromX=searchFromX,
                               section=(y, half)) for y in ys}


def runToBreaking(case, sums, endTime: float, trackInterval: float = 0.01, maxSteps: int = 1 << 40,
                  onDevice: bool = True, trackers: dict | None = None, shortestLength: float | None = None):
    """Step the case on the device from its start until the (first section's) breaking point is final
    or `endTime`, updating the trackers every `trackInterval` sqrt(d / g) of simulated time
    (src/pysurf/BreakingWave.py:885-912; src/pysurf/BreakingWave3D.py:740-770): from the device's
    reductions (`onDevice`), else from the pulled fluid positions.  `sums` holds the pushed state; a 3D
    case's trackers are its sections' (`sectionTrackers`, or `trackers`).  Returns (tracker, time,
    steps), the tracker the first section's in 3D."""
    depth = float(case.info['depth'])
    interval = trackInterval * math.sqrt(depth / 9.80665)
    if trackers is None:
        trackers = sectionTrackers(case) if case.dimensions == 3 else {None: trackerFor(case)}
    first = next(iter(trackers.values()))
    shortest = case.smoothingLength if shortestLength is None else shortestLength
    positions = None
    time, step, dt = 0.0, 0, 0.0
    nextTrack = interval
    while time < endTime and not first.breakingFinal and step < maxSteps:
        target = min(nextTrack, endTime)
        time, step, dt = sums.advance(time, step, target, maxSteps, shortest, case.cflNumber,
                                      case.maxTimeStep, case.densityFilterInterval, dt)
        if time >= nextTrack:
            if onDevice:
                for tracker in trackers.values():
                    tracker.updateOnDevice(time, sums)
            else:
                state = sums.pullState() if case.dimensions == 3 else None
                if state is not None:
                    fluidPositions = state['positions'][state['isFluid']]
                else:
                    positions = sums.pullPositions(positions)
                    fluidPositions = positions[np.asarray(case.state.isFluid, dtype=bool)]
                for tracker in trackers.values():
                    tracker.update(time, tracker.sectionOf(fluidPositions))
            nextTrack += interval
    return first, time, step
