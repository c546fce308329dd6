"""Many independent cases on one GPU: a batched parameter sweep and a served stream of solves.

A case is small beside a B200: a 2D beach of 10k-130k particles fills a fraction of the SMs, and its
run is broken every few steps by the breaking tracker's reads.  Running cases one after another
leaves the GPU mostly idle; running several at once lets one case's kernels fill the gaps of the
others'.  Each case here has its own `PairSums` (its own device state, CUDA graphs and non-blocking
stream) and its own host thread, so the cases' work overlaps on the device while their trackers
take turns on the host.  A case's result does not depend on what runs beside it: its kernels,
their order and its summation order are its own, so it is the same, bit for bit, alone and in the
mix.

    drawSweep        the 256-case sweep of 2D solitary waves on plane beaches: slope log-uniform in
                     [1/35, 1/8], H/d uniform in [0.2, 0.6], 16 to 64 particles per depth, from a seed
    solveCase        one case from its start to its breaking point (or its horizon)
    BatchRunner      cases in `slots` concurrent slots, admitted as slots and device memory free up
    serve            a stream of requests with arrival times: continuous batching, each request
                     admitted when a slot and memory are free, its latency from arrival to result
"""
from __future__ import annotations

import math
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

BYTES_PER_PARTICLE_2D = 1200        # master, frame, sort scratch and a 152-entry neighbour row
BYTES_PER_PARTICLE_3D = 5200        # the same with a ~1150-entry row


@dataclass(frozen=True)
class CaseSpec:
    """One beach case: slope, wave height over depth, particles per depth, and a solve horizon."""
    index: int
    slope: float
    height: float
    ppd: int
    endTime: float = 12.0
    toBreaking: bool = True
    scale: float = 1.0              # a 3D request's tank, scaled from 40 d x 10 d


@dataclass
class CaseResult:
    index: int
    spec: CaseSpec
    fluidParticles: int = 0
    particles: int = 0
    steps: int = 0
    simulatedTime: float = 0.0
    breakingTime: float = float('nan')
    breakingCrestX: float = float('nan')
    breakingHeight: float = float('nan')
    started: float = 0.0          # seconds on the runner's clock
    finished: float = 0.0
    error: str | None = None

    @property
    def seconds(self) -> float:
        return self.finished - self.started

    def key(self) -> tuple:
        """What must be the same alone and in the mix."""
        return (self.steps, self.simulatedTime, self.breakingTime, self.breakingCrestX, self.breakingHeight)


def drawSweep(count: int = 256, seed: int = 0, minPpd: int = 16, maxPpd: int = 64) -> list[CaseSpec]:
    """The batched sweep's cases, drawn from a seed: slope log-uniform in [1/35, 1/8], H/d uniform
    in [0.2, 0.6], particles per depth uniform over the integers minPpd..maxPpd."""
    rng = np.random.default_rng(seed)
    slopes = np.exp(rng.uniform(math.log(1.0 / 35.0), math.log(1.0 / 8.0), count))
    heights = rng.uniform(0.2, 0.6, count)
    ppds = rng.integers(minPpd, maxPpd + 1, count)
    return [CaseSpec(k, float(slopes[k]), float(heights[k]), int(ppds[k])) for k in range(count)]


def buildCase(spec: CaseSpec):
    from pysurf_b200 import cases
    return cases.solitaryBeach(spec.ppd, height=spec.height, slope=spec.slope)


def estimatedBytes(particles: int, dimensions: int = 2) -> int:
    """Device memory a case of this many particles takes, for admission."""
    return int(particles) * (BYTES_PER_PARTICLE_2D if dimensions == 2 else BYTES_PER_PARTICLE_3D) + (64 << 20)


def solveCase(spec: CaseSpec, device: int = 0, clock=time.perf_counter, case=None, tuning=None) -> CaseResult:
    """One case on the device from its start to its breaking point (the tracker's, read on the
    device every 0.01 sqrt(d / g)) or to its horizon, with the autotuner's `tuning` when one is given
    (cells per support and threads per particle; the defaults otherwise)."""
    from pysurf_b200 import breaking, cases
    result = CaseResult(spec.index, spec, started=clock())
    try:
        case = case if case is not None else buildCase(spec)
        result.fluidParticles, result.particles = case.fluidCount, case.state.nParticles
        sums = cases.pairSumsFor(case, device=device)
        if tuning is not None:
            tuning.apply(sums)
        state = case.state.copy()
        sums.push(state)
        sums.setBoundary(case.boundary, state)
        if spec.toBreaking:
            tracker, t, steps = breaking.runToBreaking(case, sums, endTime=spec.endTime)
            point = tracker.breakingPoint
            if point is not None:
                result.breakingTime, result.breakingCrestX = point.time, point.crestX
                result.breakingHeight = point.crestHeight
        else:
            t, steps, _ = sums.advance(0.0, 0, spec.endTime, 1 << 40, case.smoothingLength, case.cflNumber,
                                       case.maxTimeStep, case.densityFilterInterval)
        result.steps, result.simulatedTime = steps, t
        del sums
    except Exception as error:      # a failed case is reported with its result, the others go on
        result.error = f'{type(error).__name__}: {error}'
    result.finished = clock()
    return result


class MemoryGate:
    """Admits work while the bytes it holds fit in a budget (waiting otherwise); a request larger
    than the whole budget is admitted alone."""

    def __init__(self, budget: int):
        self.budget, self.held = int(budget), 0
        self._cond = threading.Condition()

    def acquire(self, nbytes: int) -> None:
        with self._cond:
            while self.held > 0 and self.held + nbytes > self.budget:
                self._cond.wait()
            self.held += nbytes

    def release(self, nbytes: int) -> None:
        with self._cond:
            self.held -= nbytes
            self._cond.notify_all()


def deviceBudget(device: int = 0, share: float = 0.8) -> int:
    """A share of the device memory free now."""
    import torch
    free, _ = torch.cuda.mem_get_info(device)
    return int(free * share)


@dataclass
class BatchRunner:
    """Cases in `slots` concurrent slots on one device, each admitted when a slot is free and its
    estimated memory fits the budget.  With a `tuner`, every size class among the cases is tuned
    before the first case starts, and each case runs with its class's choice."""
    slots: int = 16
    device: int = 0
    budget: int | None = None
    tuner: object = None
    results: list = field(default_factory=list)

    def run(self, specs: list[CaseSpec], builder=buildCase) -> list[CaseResult]:
        if self.tuner is not None:
            self.tuner.prepare(specs, builder)
        gate = MemoryGate(self.budget if self.budget is not None else deviceBudget(self.device))
        start = time.perf_counter()
        clock = lambda: time.perf_counter() - start     # noqa: E731

        def one(spec):
            case = builder(spec)
            need = estimatedBytes(case.state.nParticles, case.dimensions)
            tuning = self.tuner.choose(case) if self.tuner is not None else None
            gate.acquire(need)
            try:
                return solveCase(spec, self.device, clock, case, tuning)
            finally:
                gate.release(need)

        with ThreadPoolExecutor(max_workers=max(1, self.slots)) as pool:
            self.results = list(pool.map(one, specs))
        return self.results


@dataclass(frozen=True)
class Request:
    arrival: float                  # seconds after the stream starts
    spec: CaseSpec
    builder: object = None          # builds the request's case; None for a beach from the spec


def serve(requests: list[Request], slots: int = 16, device: int = 0, budget: int | None = None,
          tuner=None) -> dict:
    """Serve a stream of requests: each is admitted at its arrival, or later when a slot and memory
    are free, and solved beside the others in flight (continuous batching: a request that arrives
    while others run joins them as soon as it can).  A `tuner` supplies each request's choice from
    the classes it was prepared for (it does not time while the stream runs).  Returns the results
    with each request's latency from arrival to result, and the stream's p50/p99 latency and
    throughput."""
    gate = MemoryGate(budget if budget is not None else deviceBudget(device))
    start = time.perf_counter()
    clock = lambda: time.perf_counter() - start     # noqa: E731
    lock = threading.Lock()
    done = []

    def one(request):
        wait = request.arrival - clock()
        if wait > 0:
            time.sleep(wait)
        case = (request.builder or buildCase)(request.spec)
        need = estimatedBytes(case.state.nParticles, case.dimensions)
        tuning = tuner.choose(case) if tuner is not None else None
        gate.acquire(need)
        try:
            result = solveCase(request.spec, device, clock, case, tuning)
        finally:
            gate.release(need)
        with lock:
            done.append((request, result))

    ordered = sorted(requests, key=lambda r: r.arrival)
    with ThreadPoolExecutor(max_workers=max(1, slots)) as pool:
        list(pool.map(one, ordered))
    total = clock()
    latencies = np.array([result.finished - request.arrival for request, result in done])
    updates = sum(result.fluidParticles * result.steps for _, result in done)
    return {'results': [result for _, result in sorted(done, key=lambda d: d[1].index)],
            'latency_p50_s': float(np.percentile(latencies, 50)) if len(latencies) else float('nan'),
            'latency_p99_s': float(np.percentile(latencies, 99)) if len(latencies) else float('nan'),
            'seconds': total, 'particle_updates_per_s': updates / total if total > 0 else float('nan')}


def poissonArrivals(count: int, rate: float, seed: int = 0) -> np.ndarray:
    """Arrival times of a Poisson stream of `rate` requests a second."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, count))
