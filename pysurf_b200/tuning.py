"""The autotuner: a case's cell size and threads per particle, picked by timing device steps.

Two settings of the device step change its speed and not its physics:

    cells per support     the cell list's cells are 2h / c wide (c = 1..4).  Finer cells offer fewer
                          candidates outside the support, for a stencil of more cells to walk.
    threads per particle  how many threads share one particle's neighbours in the sweeps (1, 2, 4 or
                          8).  More threads put more loads in flight for a small case; fewer spend
                          fewer shuffles combining the partial sums of a large one.

Which pair is fastest depends on the case's size and its neighbour count, so the tuner times them on
the device: each candidate runs a few warm-up steps and then `steps` timed steps from the case's
start (device events around the steps, `PairSums.lastAdvanceMilliseconds`), and the one with the
fewest milliseconds a step wins.

A choice changes the order the sweeps add a particle's neighbours in, so results under two choices
differ in their last bits (each stays within the step's float32 tolerance of the float64 oracle).
For that reason a batch decides every choice before its first case starts: `Autotuner.prepare` sorts
the cases into size classes (dimensions, kernel and half-octaves of the particle count) and times one
case of middle size per class; each case then runs with its class's choice, the same whether it runs
alone or beside others.  Choices can be saved to and loaded from a JSON file, so a sweep that is run
again takes the same ones without timing.

    Tuning        one choice (cells per support, threads per particle)
    candidates    the choices tried for a dimension
    timeTuning    milliseconds a step of one case under one choice
    tuneCase      every candidate timed on one case; the fastest and the whole table
    Autotuner     choices by size class: prepared before a batch, looked up per case, saved as JSON
"""
from __future__ import annotations

import json
import math
from dataclasses import asdict, dataclass, field

DEFAULT_CELLS = 3
DEFAULT_THREADS = 4


@dataclass(frozen=True)
class Tuning:
    cellsPerSupport: int = DEFAULT_CELLS
    threadsPerParticle: int = DEFAULT_THREADS

    def apply(self, sums) -> None:
        """Set this choice on a PairSums (before its push: the cell list is rebuilt for it)."""
        sums.setCellsPerSupport(self.cellsPerSupport)
        sums.setSweepOptions(True, self.threadsPerParticle)


def candidates(dimensions: int) -> list[Tuning]:
    """The choices tried: 2D cases have about 110 neighbours at h = 3 dx, so every thread count up to 8
    has work; 3D cases have about 850, where one or two threads a particle leave too few in flight."""
    if dimensions == 2:
        return [Tuning(c, t) for c in (2, 3, 4) for t in (2, 4, 8)]
    return [Tuning(c, t) for c in (2, 3) for t in (4, 8)]


def sizeClass(dimensions: int, kernelType: str, particles: int) -> str:
    """Cases of one dimension and kernel whose particle counts share a half-octave."""
    return f'{dimensions}d-{kernelType}-{int(math.floor(2.0 * math.log2(max(int(particles), 1))))}'


def timeTuning(case, tuning: Tuning, steps: int = 20, warmup: int = 3, device: int = 0) -> float:
    """Milliseconds a device step of `case` takes under `tuning`: `warmup` steps from the case's start
    (the first builds the cell list and the neighbour table and captures the step's graphs), then
    `steps` steps timed with device events."""
    from pysurf_b200 import cases
    sums = cases.pairSumsFor(case, device=device)
    tuning.apply(sums)
    state = case.state.copy()
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    args = (case.smoothingLength, case.cflNumber, case.maxTimeStep, case.densityFilterInterval)
    t, s, dt = sums.advance(0.0, 0, math.inf, warmup, *args)
    t, s, dt = sums.advance(t, s, math.inf, warmup + steps, *args, lastTimeStep=dt)
    ms = sums.lastAdvanceMilliseconds()
    del sums
    return ms / steps


@dataclass
class TuneResult:
    best: Tuning
    milliseconds: dict          # Tuning -> ms a step

    def table(self) -> list:
        return [{**asdict(k), 'ms_per_step': v} for k, v in sorted(self.milliseconds.items(), key=lambda kv: kv[1])]


def tuneCase(case, steps: int = 20, warmup: int = 3, device: int = 0, timer=timeTuning,
             choices: list[Tuning] | None = None) -> TuneResult:
    """Time every candidate on one case; the fastest wins, ties going to the earlier candidate."""
    choices = choices if choices is not None else candidates(case.dimensions)
    if not choices:
        raise ValueError('no candidates to time')
    times = {}
    for choice in choices:
        ms = float(timer(case, choice, steps=steps, warmup=warmup, device=device))
        if not (ms > 0.0 and math.isfinite(ms)):
            raise RuntimeError(f'timing {choice} gave {ms} ms a step')
        times[choice] = ms
    best = min(choices, key=lambda c: times[c])
    return TuneResult(best, times)


@dataclass
class Autotuner:
    """Choices by size class.  `prepare` times one case per class not yet known; `choose` looks a case's
    class up and falls back to the default choice for a class never prepared (it never times, so a
    choice cannot depend on what else runs)."""
    steps: int = 20
    warmup: int = 3
    device: int = 0
    timer: object = timeTuning
    choices: dict = field(default_factory=dict)     # size class -> Tuning
    tables: dict = field(default_factory=dict)      # size class -> TuneResult.table()

    @staticmethod
    def classOf(case) -> str:
        return sizeClass(case.dimensions, case.kernelType, case.state.nParticles)

    def prepare(self, items, builder=None) -> dict:
        """Time a middle-sized case of every size class among `items` (cases, or specs that `builder`
        turns into cases) that has no choice yet.  Returns the classes tuned now with their tables."""
        items = list(items)     # walked twice: a generator would be spent by the first walk
        sizes = {}
        for k, item in enumerate(items):
            case = builder(item) if builder is not None else item
            sizes.setdefault(self.classOf(case), []).append((case.state.nParticles, k))
        tuned = {}
        for key in sorted(sizes):
            if key in self.choices:
                continue
            members = sorted(sizes[key])
            _, k = members[len(members) // 2]
            case = builder(items[k]) if builder is not None else items[k]
            result = tuneCase(case, self.steps, self.warmup, self.device, self.timer)
            self.choices[key] = result.best
            self.tables[key] = result.table()
            tuned[key] = self.tables[key]
        return tuned

    def choose(self, case) -> Tuning:
        return self.choices.get(self.classOf(case), Tuning())

    def save(self, path: str) -> None:
        with open(path, 'w') as f:
            json.dump({'choices': {k: asdict(v) for k, v in self.choices.items()}, 'tables': self.tables}, f,
                      indent=1, sort_keys=True)

    def load(self, path: str) -> None:
        with open(path) as f:
            data = json.load(f)
        for k, v in data.get('choices', {}).items():
            choice = Tuning(int(v['cellsPerSupport']), int(v['threadsPerParticle']))
            if choice.cellsPerSupport not in (1, 2, 3, 4) or choice.threadsPerParticle not in (1, 2, 4, 8):
                raise ValueError(f'{path}: class {k} has an invalid choice {choice}')
            self.choices[k] = choice
        self.tables.update(data.get('tables', {}))
