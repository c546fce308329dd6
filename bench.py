"""Benchmark: fluid particle-updates/s of the deltaSph step on the 3D solitary wave over a Gaussian ridge.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--case ridge|beach] [--ppd P]

Workload (the default): a first-order solitary wave of H/d = 0.5 crossing a Gaussian ridge (0.6 d
high, sigma 3 d, its axis at 25 degrees to the crest) in a walled 40 d x 10 d tank, 32 particles
per depth (pysurf_b200.cases.ridgeWave3D, 11.7M fluid and 4.1M boundary particles), whose crest zone
(every column whose surface stands 0.3 H above still water) is split on the device into 8 daughters
of h / 2 before the timing: 22.9M fluid particles.  Stepped by the deltaSph scheme (Wendland C2 at
h = 3 dx, hydrostatic delta-SPH diffusion, the continuity correction, extrapolated walls, the
viscosity limiter, density floor 0.9 rho0).  A step is one full device-resident step: cell list and
neighbour table over both grid levels, wall pressure, gradients, momentum, time step, kick,
continuity, density update, drift and height-field enforcement.  --no-refine skips the split;
--case beach steps the 2D solitary wave of H/d = 0.45 over a 1:15 beach at 64 particles per depth
(pysurf_b200.cases.solitaryBeach) instead.

value      fluid particles x steps / device time of exactly K steps (CUDA events on the stream the
           kernels run on, an L2 flush of 256 MiB between steps outside the timed spans), max over
           ranks; with N GPUs each rank runs its own replica of the case (independent cases need
           no collective), so the value is the sum over replicas ("scaling": "weak").
e2e        the same metric through the public API with host buffers: each step pushes the whole
           state (after the split: its lengths too) from pinned host memory, steps once and pulls
           the state back.
roofline   the dominant kernel (momentum) against the measured HBM copy bandwidth, with the
           step's algorithmic bytes per fluid particle-update (53 B in 2D, 69 B in 3D, 4 B more
           with mixed smoothing lengths) per launch.
pair_flops the three sweeps' float32 work, 150 flop a directed pair, against the nominal FP32 SIMT
           peak: the gather sweeps are bound by latency and issue, not by HBM.
cpu_baseline and --impl reference   the float64 C restatement of the reference's step (oracle/,
           OpenMP over every host core), timed per step: on the beach over the whole case; on the
           ridge over a sample of it, the particles of a slab of whole columns across the tank's
           middle (y within 0.125 d of it) over the tank's full length, split by the same zone rule,
           since a float64 step over all 27M particles takes minutes.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# algorithmic bytes per fluid particle-update: read x (offset + cell), v, rho, m, kind; write x, v, rho
ALGORITHMIC_BYTES = {2: 53, 3: 69}
FLOP_PER_PAIR = 150             # float32 flop per directed pair per step over the three sweeps (gradients,
                                # momentum with the limiter, continuity with diffusion)
FP32_SIMT_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12   # nominal: 148 SMs x 128 FP32 lanes x FMA x 1965 MHz
METRIC = 'particle-updates/s'


def parseArgs():
    p = argparse.ArgumentParser()
    p.add_argument('--gpus', type=int, default=1)
    p.add_argument('--steps', type=int, default=40)
    p.add_argument('--warmup', type=int, default=5)
    p.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    p.add_argument('--case', default='ridge', choices=['ridge', 'beach'],
                   help='ridge: the 3D Gaussian ridge, crest zone split (the headline); beach: the 2D solitary wave '
                        'on a 1:15 beach')
    p.add_argument('--ppd', type=int, default=None, help='particles per depth (32 ridge, 64 beach)')
    p.add_argument('--cells', type=int, default=None, help='cells per kernel support in the device cell list')
    p.add_argument('--threads', type=int, default=None, help='threads per particle in the sweeps (1, 2, 4, 8)')
    p.add_argument('--no-table', action='store_true', help='walk the cells in every sweep (no neighbour table)')
    p.add_argument('--to-breaking', action='store_true',
                   help='run the beach from its start to the breaking point and report the time it takes')
    p.add_argument('--sweep', type=int, default=0,
                   help='solve this many cases of the seeded 256-case beach sweep to their breaking points, '
                        'case by case and then batched, and report both')
    p.add_argument('--slots', type=int, default=16, help='concurrent cases in the batched sweep and the server')
    p.add_argument('--no-serial', action='store_true',
                   help='batched sweep: skip the case-by-case run (the line then has no speed-up)')
    p.add_argument('--tune', action='store_true',
                   help='batched sweep: pick each size class\'s cells per support and threads per particle by '
                        'timing (the autotuner, its time counted in the batched run)')
    p.add_argument('--serve', type=int, default=0,
                   help='serve this many requests arriving as a Poisson stream (see serveBench)')
    p.add_argument('--horizon-scale', type=float, default=0.1,
                   help='the served requests horizons, U(2, 6) s of simulated time times this')
    p.add_argument('--rate', type=float, default=20.0, help='the served stream\'s arrivals a second')
    p.add_argument('--no-refine', action='store_true',
                   help='ridge: leave the crest zone (surface above 0.3 H) whole instead of splitting it into '
                        'daughters of h/2 before the timing')
    p.add_argument('--options', default='',
                   help='opt-in parts of the step, comma separated: closure (delta-LES-SPH), shifting, energy '
                        '(the energy budget), compensated (compensated momentum and continuity sums)')
    p.add_argument('--no-e2e', action='store_true')
    p.add_argument('--no-cpu', action='store_true')
    return p.parse_args()


OPTIONS = ('closure', 'shifting', 'energy', 'compensated')


def buildCase(args):
    from pysurf_b200 import cases
    case = cases.ridgeWave3D(args.ppd or 32) if args.case == 'ridge' else cases.solitaryBeach(args.ppd or 64)
    options = [o for o in args.options.split(',') if o]
    unknown = set(options) - set(OPTIONS)
    if unknown:
        raise SystemExit(f'unknown --options {sorted(unknown)}; choose from {OPTIONS}')
    case.turbulenceClosure = 'deltaLes' if 'closure' in options else case.turbulenceClosure
    case.particleShifting = 'shifting' in options or case.particleShifting
    case.trackEnergy = 'energy' in options or case.trackEnergy
    case.compensatedSums = 'compensated' in options or case.compensatedSums
    case.info['options'] = options
    return case


def config(case, flush: bool = True) -> dict:
    info = dict(case.info)
    scheme = ('deltaSph scheme (Wendland C2 h=3dx, hydrostatic delta-SPH 0.1, continuity correction, extrapolated '
              'walls, viscosity limiter)')
    if case.dimensions == 2:
        workload = f'solitary wave H/d 0.45 on a 1:15 plane beach, 2D, {scheme}'
        extent = {'domain_length_d': info['length']}
    else:
        workload = (f'solitary wave H/d 0.5 over a Gaussian ridge (0.6 d, sigma 3 d, axis at 25 degrees) in a '
                    f'40 d x 10 d tank, 3D, {scheme}')
        extent = {'tank_d': info['tank']}
    if info.get('options'):
        workload += ', with ' + ' and '.join({'closure': 'the delta-LES-SPH closure', 'shifting': 'particle shifting',
                                               'energy': 'the energy budget',
                                               'compensated': 'compensated momentum and continuity sums'}[o]
                                              for o in info['options'])
    return {'workload': workload, 'particles_per_depth': info['ppd'], 'fluid_particles': case.fluidCount,
            'boundary_particles': int(case.state.nParticles - case.fluidCount), 'boundary_layers': info['layers'],
            'smoothing_length_over_dx': round(case.smoothingLength / case.spacing, 6), **extent,
            'l2': 'flushed (256 MiB write) between timed steps' if flush else 'resident'}


def meanNeighbours(case, sample: int = 20000) -> float:
    """Neighbours within 2h of a fluid particle at the start, the mean over a seeded sample, for the
    pair-flop figure."""
    import numpy as np
    from scipy.spatial import cKDTree
    positions = case.state.positions
    fluid = np.flatnonzero(case.state.isFluid)
    chosen = np.random.default_rng(0).choice(fluid, size=min(sample, fluid.size), replace=False)
    counts = cKDTree(positions).query_ball_point(positions[chosen], 2.0 * case.smoothingLength, return_length=True)
    return float(np.mean(counts) - 1.0)


RIDGE_SAMPLE_HALF_WIDTH = 0.125    # d: the ridge's CPU sample is the columns within this of the tank's middle


def refines(case, args) -> bool:
    return case.dimensions == 3 and not args.no_refine


def ridgeSample(case, refine: bool, halfWidth: float = RIDGE_SAMPLE_HALF_WIDTH) -> dict:
    """A bounded sample of the ridge workload for the float64 CPU step: every particle (fluid, bed and
    end walls) of the columns -- one spacing across, as the crest zone counts them -- within halfWidth d
    of the tank's middle line in y, over the tank's full length, split by the device's zone rule
    (oracle.crestZone, then oracle.splitParticles into 8 daughters of h / 2).  The slab's particles near
    its y edges miss the neighbours beyond them, so a float64 step over it costs less a particle than
    over the whole tank.  Also the mean neighbour count (r < h_i + h_j) of the slab's fluid, counted
    among the particles of a slab two supports wider, as in the whole tank."""
    import numpy as np
    from scipy.spatial import cKDTree
    from oracle import oracle
    st, s, info = case.state, case.spacing, case.info
    lower, upper = case.domainMin, case.domainMax
    nx = int(math.ceil((upper[0] - lower[0]) / s))
    ny = int(math.ceil((upper[1] - lower[1]) / s))
    rows = int(round(halfWidth * float(info['depth']) / s))
    margin = int(math.ceil(4.0 * case.smoothingLength / s))
    centre = int(math.floor((0.5 * float(info['tank'][1]) - lower[1]) / s + 0.5))
    cy = np.floor((st.positions[:, 1] - lower[1]) / s)
    keep = (cy >= centre - rows - margin) & (cy < centre + rows + margin)
    wide = {'positions': st.positions[keep].copy(), 'velocities': st.velocities[keep].copy(),
            'densities': st.densities[keep].copy(), 'masses': np.broadcast_to(st.masses, keep.shape)[keep].copy(),
            'isFluid': st.isFluid[keep].copy(), 'lengths': np.full(int(keep.sum()), case.smoothingLength)}
    if refine:
        depth, height = float(info['depth']), float(info['H/d']) * float(info['depth'])
        fluidMass = float(np.max(st.masses[st.isFluid]))
        zone = oracle.crestZone(wide, lower[0], lower[1], s, nx, ny, depth + 0.3 * height, 0.999 * fluidMass)
        oracle.splitParticles(wide, zone, case.referenceDensity, case.smoothingLength, 0.5)
    x, h = wide['positions'], wide['lengths']
    column = np.floor((x[:, 1] - lower[1]) / s)
    narrow = (column >= centre - rows) & (column < centre + rows)
    fluid = np.flatnonzero(narrow & wide['isFluid'])
    chosen = np.random.default_rng(0).choice(fluid, size=min(20000, fluid.size), replace=False)
    tree, hmax = cKDTree(x), float(h.max())
    counts = []
    for i, near in zip(chosen, tree.query_ball_point(x[chosen], h[chosen] + hmax)):
        near = np.asarray(near)
        r = np.linalg.norm(x[near] - x[i], axis=1)
        counts.append(int(np.count_nonzero(r < h[i] + h[near])) - 1)
    sample = {k: v[narrow] for k, v in wide.items()}
    sample['neighbours'] = float(np.mean(counts)) if counts else float('nan')
    sample['description'] = (f'the columns within {halfWidth} d of the tank\'s middle over its full length '
                             f'({int(sample["isFluid"].sum())} fluid and {int((~sample["isFluid"]).sum())} boundary '
                             f'particles{", crest zone split" if refine else ""})')
    return sample


def oracleStepper(case):
    """The float64 C restatement of the device step (oracle/) set up for the case."""
    from oracle import oracle
    boundary = case.boundary
    if type(boundary).__name__ == 'BedBoundary':
        bed = boundary.bathymetry
        enforcement = ('bed', oracle.bedParams(bed.x, bed.z, 0.25 * case.spacing, False, 0.0, True, bed.startX, 0.0,
                                               bed.endX))
    else:
        field, clearance = boundary.field, 0.25 * boundary.spacing
        startX, endX, startY, endY = field.bounds
        enforcement = ('field', oracle.fieldParams(field.z, field.x[0], field.y[0], field.spacingX, field.spacingY,
                                                   clearance, startY + clearance, endY - clearance, True,
                                                   startX + clearance, endX - clearance))
    stepper = oracle.Stepper(case.dimensions, case.kernelType, case.smoothingLength, case.referenceDensity,
                             case.soundSpeed, case.alpha, case.gravity, 0.0, 0.0, case.densityFloor,
                             case.densityDiffusion, case.diffusionDelta, True, False, True, True, case.cflNumber,
                             case.maxTimeStep, 0.0, 0, enforcement, closure=case.turbulenceClosure == 'deltaLes',
                             viscosity=case.kinematicViscosity, shifting=case.particleShifting,
                             shiftingMach=case.shiftingMach, spacing=case.spacing, shiftingLocal=case.shiftingLocal)
    if case.trackEnergy:
        stepper.trackEnergy()
    return stepper


def sweepConfig(sums, table: bool, threads: int) -> dict:
    return {'cells_per_support': sums.cellsPerSupport, 'threads_per_particle': threads, 'neighbour_table': table,
            'table_row_capacity': sums.neighborTableCapacity()}


def clockSampler(device: int):
    """nvidia-smi clocks and throttle reasons every 200 ms while the timed region runs."""
    samples, stop = [], threading.Event()

    def run():
        query = ('clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,'
                 'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
                 'clocks_event_reasons.sw_power_cap')
        while not stop.is_set():
            try:
                out = subprocess.run(['nvidia-smi', '-i', str(device), f'--query-gpu={query}',
                                      '--format=csv,noheader,nounits'], capture_output=True, text=True, timeout=5)
                fields = [f.strip() for f in out.stdout.strip().split(',')]
                if len(fields) == 7:
                    samples.append(fields)
            except Exception:
                pass
            stop.wait(0.2)

    thread = threading.Thread(target=run, daemon=True)
    thread.start()

    def finish():
        stop.set()
        thread.join(timeout=10)
        if not samples:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['unsampled']}
        sm = sorted(float(s[0]) for s in samples if s[0].replace('.', '').isdigit())
        reasons = set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for s in samples:
            for name, value in zip(names, s[3:]):
                if value.lower().startswith('active'):
                    reasons.add(name)
        return {'sm_mhz': sm[len(sm) // 2] if sm else None, 'sm_max_mhz': float(samples[0][1]),
                'reasons': sorted(reasons), 'samples': len(samples)}

    return finish


def measuredPeaks() -> dict:
    path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
        return {'hbm_gbs': float(data['hbm_gbs']), 'source': 'measured'}
    return {'hbm_gbs': 6650.0, 'source': 'fallback'}


def profiledTraffic(case, kernel: str, refined: bool, fluid: int) -> float | None:
    """DRAM bytes a launch of `kernel` (gradients, momentum, continuity) from the committed ncu summary of
    this workload: the beach at its own size; the refined ridge captured at 12 ppd (the bench's size
    is too large to capture), whose traffic -- the neighbour table, which grows with the particles --
    is scaled to this run by its fluid particles after the split."""
    if case.dimensions == 2:
        name = 'sweeps_solitaryBeach64.md'
    elif refined:
        name = 'sweeps_ridgeWave3D12_refined.md'
    else:
        return None
    path = os.path.join(ROOT, 'profiles', name)
    if not os.path.exists(path):
        return None
    text = open(path).read()
    match = re.search(rf'traffic_bytes_per_launch_{kernel}:\s*([0-9.eE+]+)', text)
    captured = re.search(r'fluid_particles:\s*([0-9]+)', text)
    if not match or not captured:
        return None
    return float(match.group(1)) * fluid / float(captured.group(1))


def cpuState(case, refine: bool) -> tuple:
    """The state the float64 CPU step runs on, its fluid count and what it is: the whole beach, or the
    ridge's sample (ridgeSample)."""
    import numpy as np
    if case.dimensions == 3:
        sample = ridgeSample(case, refine)
        return sample, int(sample['isFluid'].sum()), 'one float64 step over a sample of the workload: ' + \
            sample.pop('description')
    state = {k: np.array(getattr(case.state, k), copy=True) for k in ('positions', 'velocities', 'densities',
                                                                       'masses', 'isFluid')}
    return state, case.fluidCount, f'full steps of the whole case ({case.state.nParticles} particles) in float64'


def cpuBaseline(case, refine: bool, seconds: float = 12.0) -> dict:
    """The float64 oracle's step on the same workload (the ridge: its sample), on every host core, for
    about `seconds` after one untimed step."""
    stepper = oracleStepper(case)
    state, fluid, what = cpuState(case, refine)
    state.pop('neighbours', None)
    stepper(state)                          # warm-up: page in, first neighbour list
    steps, start = 0, time.perf_counter()
    while True:
        stepper(state)
        steps += 1
        elapsed = time.perf_counter() - start
        if elapsed > seconds or steps >= 200:
            break
    cores = os.cpu_count()
    return {'value': fluid * steps / elapsed, 'unit': METRIC, 'cores': cores, 'kind': 'port',
            'sample': f'{steps} x {what}, OpenMP over {cores} threads, {elapsed:.1f} s'}


def referenceArm(args) -> None:
    """The reference's algorithm on the host cores: the float64 C restatement (oracle/), timed per step
    (the ridge: each step over its sample)."""
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return
    case = buildCase(args)
    refine = refines(case, args)
    stepper = oracleStepper(case)
    state, fluid, what = cpuState(case, refine)
    state.pop('neighbours', None)
    for _ in range(args.warmup):
        stepper(state)
    start = time.perf_counter()
    for _ in range(args.steps):
        stepper(state)
    elapsed = time.perf_counter() - start
    value = fluid * args.steps / elapsed
    cores = os.cpu_count()
    line = {'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': METRIC, 'n_gpus': args.gpus,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': 1e3 * elapsed / args.steps,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
            'config': dict(config(case, flush=False), crest_zone_split=refine),
            'cpu_baseline': {'value': value, 'unit': METRIC, 'cores': cores, 'kind': 'port',
                             'sample': f'{args.steps} x {what}, OpenMP over {cores} threads'},
            'e2e': {'value': value, 'unit': METRIC, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)


def toBreaking(args) -> None:
    """The case from its start to the breaking point on one GPU: the device steps, with the breaking
    tracker (the ridge: its middle section's) reading the wave on the device every 0.01 sqrt(d / g)
    (what the reference's facades do, src/pysurf/BreakingWave.py:885-912); wall time from push to the
    breaking point."""
    import torch
    from pysurf_b200 import breaking, cases
    case = buildCase(args)
    sums = cases.pairSumsFor(case, args.cells)
    sums.setSweepOptions(not args.no_table, args.threads or 4)
    state = case.state.copy()
    torch.cuda.synchronize()
    start = time.perf_counter()
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    shortest = case.smoothingLength
    if refines(case, args):
        cases.refineCrestZone(sums, case)
        shortest *= 0.5
    # the ridge's sections, or the beach's tracker; the 32-ppd ridge takes hours to its breaking point
    tracker, simulated, steps = breaking.runToBreaking(case, sums, endTime=12.0, shortestLength=shortest)
    torch.cuda.synchronize()
    wall = time.perf_counter() - start
    point = tracker.breakingPoint
    line = {'metric': 'seconds to the breaking point', 'value': wall, 'unit': 's', 'n_gpus': 1,
            'higher_is_better': False, 'data': 'synthetic', 'config': config(case, flush=False),
            'steps': steps, 'simulated_time_s': simulated, 'tracker_updates': len(tracker.times),
            'particle_updates_per_s': case.fluidCount * steps / wall,
            'breaking': None if point is None else {
                'time_s': point.time, 'crest_x': point.crestX, 'Hb_over_d': point.crestHeight / case.info['depth'],
                'hb_over_d': point.depth / case.info['depth'], 'lean': point.lean}}
    print(json.dumps(line), flush=True)


def sweepBench(args) -> None:
    """The batched sweep at the size asked: the first --sweep cases of the seeded sweep (slope
    log-U(1/35, 1/8), H/d U(0.2, 0.6), 16-64 ppd) to their breaking points, first one after another
    (unless --no-serial), then --slots at a time.  Untuned, every batched result must equal its
    case-by-case one bit for bit; tuned (--tune), its breaking point must lie within 1% of it."""
    import numpy as np
    from pysurf_b200 import batch
    from pysurf_b200 import tuning
    specs = batch.drawSweep(256, seed=0)[:args.sweep]
    tuner = tuning.Autotuner() if args.tune else None
    runs = {}
    arms = (('case_by_case', 1, None), ('batched', args.slots, tuner))
    for name, slots, tune in arms[1:] if args.no_serial else arms:
        start = time.perf_counter()
        results = batch.BatchRunner(slots=slots, tuner=tune).run(specs)
        runs[name] = (time.perf_counter() - start, results)
    batched, mixed = runs['batched']
    serial, alone = runs.get('case_by_case', (None, None))
    ok = all(m.error is None for m in mixed) and (alone is None or all(a.error is None for a in alone))
    if alone is None:
        check = {'errors': sum(1 for m in mixed if m.error is not None)}
        if tuner is not None:
            check['tuned_classes'] = {k: vars(v) for k, v in sorted(tuner.choices.items())}
    elif tuner is None:
        check = {'results_identical_alone_and_batched': ok and all(a.key() == m.key() for a, m in zip(alone, mixed))}
    else:
        # tuned choices add neighbours in another order: the breaking point, not the bits, must agree
        def within(a, m):
            if a.breakingTime != a.breakingTime:
                return m.breakingTime != m.breakingTime
            return (abs(m.breakingTime - a.breakingTime) <= 0.01 * a.breakingTime
                    and abs(m.breakingCrestX - a.breakingCrestX) <= 0.01 * a.breakingCrestX)
        check = {'breaking_within_1pct_of_default_case_by_case': ok and all(within(a, m) for a, m in zip(alone, mixed)),
                 'tuned_classes': {k: vars(v) for k, v in sorted(tuner.choices.items())}}
    updates = sum(r.fluidParticles * r.steps for r in mixed)
    broke = sum(1 for r in mixed if r.breakingTime == r.breakingTime)
    seconds = np.array([r.seconds for r in mixed])
    line = {'metric': 'cases/h', 'value': 3600.0 * len(specs) / batched, 'unit': 'cases/h', 'n_gpus': 1,
            'higher_is_better': True, 'data': 'synthetic',
            'config': {'workload': f'the first {len(specs)} cases of the 256-case 2D beach sweep (seed 0), each to '
                                   f'its breaking point', 'slots': args.slots, 'autotuned': bool(args.tune),
                       'fluid_particles': [r.fluidParticles for r in mixed]},
            'case_by_case_cases_per_h': 3600.0 * len(specs) / serial if serial else None,
            'speedup': serial / batched if serial else None,
            'seconds_batched': batched, 'seconds_case_by_case': serial, 'broke': broke,
            **check, 'particle_updates_per_s': updates / batched,
            'case_seconds_p50': float(np.percentile(seconds, 50)),
            'case_seconds_p99': float(np.percentile(seconds, 99))}
    print(json.dumps(line), flush=True)


RIDGE16_PARTICLES = 2469130     # the 40 d x 10 d ridge at 16 particles per depth


def ridgeRequest(spec):
    """A served 3D request: the Gaussian ridge at the spec's ppd in a tank scaled from 40 d x 10 d by
    the spec's `scale`, the crest at a fifth and the ridge at half its length."""
    from pysurf_b200 import cases
    scale = float(spec.scale)
    length, width = 40.0 * scale, 10.0 * scale
    return cases.ridgeWave3D(spec.ppd, length=length, width=width, crestX=0.2 * length, ridgeX=0.5 * length)


def serveBench(args) -> None:
    """The served stream: --serve requests arriving as a Poisson stream at --rate a second (seed 0),
    80% 2D beaches drawn as the sweep draws them (5k-130k fluid particles) and 20% 3D ridges at 16 ppd
    in tanks sized for 0.5M-4M particles, each run for U(2, 6) s of simulated time times
    --horizon-scale; admitted as slots (--slots) and device memory free up, solved beside the requests
    in flight.  Beside p50/p99 latency the line reports the load the stream offers (its particle-updates
    over its arrival span) against what the device cleared while it held a request (its particle-updates
    over the union of the requests' solve spans): offered over cleared above 1 is a queue that grows,
    and its latencies are its depth."""
    import numpy as np
    from pysurf_b200 import batch
    rng = np.random.default_rng(0)
    sweep = batch.drawSweep(args.serve, seed=0)
    arrivals = batch.poissonArrivals(args.serve, args.rate, seed=0)
    requests = []
    for k in range(args.serve):
        horizon = float(rng.uniform(2.0, 6.0)) * args.horizon_scale
        if rng.uniform() < 0.2:
            scale = math.sqrt(float(rng.uniform(0.5e6, 4.0e6)) / RIDGE16_PARTICLES)
            spec = batch.CaseSpec(k, 0.0, 0.5, 16, endTime=horizon, toBreaking=False, scale=scale)
            requests.append(batch.Request(float(arrivals[k]), spec, ridgeRequest))
        else:
            base = sweep[k]
            spec = batch.CaseSpec(k, base.slope, base.height, base.ppd, endTime=horizon, toBreaking=False)
            requests.append(batch.Request(float(arrivals[k]), spec))
    out = batch.serve(requests, slots=args.slots)
    results = out['results']
    updates = sum(r.fluidParticles * r.steps for r in results)
    span = float(arrivals[-1] - arrivals[0]) if args.serve > 1 else float('nan')
    offered = updates / span if span > 0 else float('nan')
    # the seconds with at least one request on the device: the union of the requests' solve spans
    busy, reach = 0.0, -math.inf
    for begin, end in sorted((r.started, r.finished) for r in results):
        if end > reach:
            busy += end - max(begin, reach)
            reach = end
    cleared = updates / busy if busy > 0 else float('nan')
    line = {'metric': 'p99 latency', 'value': out['latency_p99_s'], 'unit': 's', 'n_gpus': 1,
            'higher_is_better': False, 'data': 'synthetic',
            'config': {'workload': f'{args.serve} requests, Poisson {args.rate}/s, 80% 2D beach 16-64 ppd, 20% 3D '
                                   f'ridge 16 ppd 0.5M-4M particles, horizons U(2, 6) s x {args.horizon_scale}',
                       'slots': args.slots},
            'latency_p50_s': out['latency_p50_s'], 'latency_p99_s': out['latency_p99_s'],
            'seconds': out['seconds'], 'particle_updates_per_s': out['particle_updates_per_s'],
            'offered_particle_updates_per_s': offered, 'arrival_span_s': span, 'busy_s': busy,
            'cleared_while_busy_particle_updates_per_s': cleared,
            'offered_over_cleared': offered / cleared if cleared == cleared and cleared > 0 else None,
            'failed': sum(1 for r in results if r.error), 'particles': [r.particles for r in results]}
    print(json.dumps(line), flush=True)


def main() -> None:
    args = parseArgs()
    if args.serve:
        serveBench(args)
        return
    if args.sweep:
        sweepBench(args)
        return
    if args.impl == 'reference':
        referenceArm(args)
        return
    if args.to_breaking:
        toBreaking(args)
        return
    import numpy as np
    import torch

    from pysurf_b200 import cases, replicas

    ranks = replicas.ranksFromEnvironment()
    rank, world, local = ranks.rank, ranks.world, ranks.local
    torch.cuda.set_device(local)
    replicas.initialize(ranks, 'nccl')

    case = buildCase(args)
    sums = cases.pairSumsFor(case, args.cells, device=local)
    sums.setSweepOptions(not args.no_table, args.threads or 4)
    stream = torch.cuda.Stream()
    sums.setStream(stream.cuda_stream)
    state = case.state.copy()
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    h, cfl, maxdt = case.smoothingLength, case.cflNumber, case.maxTimeStep
    refine = refines(case, args)
    refined = None
    if refine:
        refined = cases.refineCrestZone(sums, case)
        h = 0.5 * case.smoothingLength     # the shortest length sets the time step
    # the 2D start's neighbour count from the whole case; the ridge's from its CPU sample (a tree over
    # every one of its particles takes longer than the run), which is split as the device split
    sample = ridgeSample(case, refine) if case.dimensions == 3 else None
    neighbours = sample['neighbours'] if sample is not None else meanNeighbours(case)
    del sample
    fluidCount = case.fluidCount + (refined or 0) * (2 ** case.dimensions - 1)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device='cuda')     # 256 MiB, twice the L2

    # warm-up steps (untimed), then exactly K timed steps
    sums.beginSteps(0.0, 0, math.inf, 1 << 62, h, cfl, maxdt)
    sums.enqueueSteps(args.warmup)
    t, s, dt = sums.finishSteps()
    sums.beginSteps(t, s, math.inf, 1 << 62, h, cfl, maxdt, lastTimeStep=dt)
    launchesPerStep = sums.stepLaunches()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stageMs = []
    replicas.barrier(ranks)
    torch.cuda.synchronize()
    sampler = clockSampler(local)
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            starts[k].record(stream)
            sums.enqueueSteps(1)
            stops[k].record(stream)
        stream.synchronize()
        stageMs.append(sums.stageTimes())
    torch.cuda.synchronize()
    clocks = sampler()
    t, s, dt = sums.finishSteps()
    stepMs = [a.elapsed_time(b) for a, b in zip(starts, stops)]
    totalMs = replicas.maxOverRanks(float(sum(stepMs)), ranks)
    replicas.barrier(ranks)
    value = world * fluidCount * args.steps / (totalMs / 1e3)

    names = sums.stageNames()
    stages = {name: float(np.mean([m[i] for m in stageMs])) for i, name in enumerate(names)}
    # the dominant single kernel: the 'cells' stage is several launches (the sort's five and the table)
    dominant = max((name for name in stages if name != 'cells'), key=stages.get)
    peaks = measuredPeaks()
    kernelMs = stages[dominant]
    unitBytes = ALGORITHMIC_BYTES[case.dimensions] + (4 if refine else 0)     # + h when the lengths are mixed
    achieved = unitBytes * fluidCount / (kernelMs / 1e3) / 1e9
    pairFlop = fluidCount * neighbours * FLOP_PER_PAIR
    simt = {'flop_per_pair': FLOP_PER_PAIR, 'neighbours_per_fluid_particle': neighbours,
            'achieved_tflops': pairFlop / (totalMs / args.steps / 1e3) / 1e12, 'peak_tflops': FP32_SIMT_TFLOPS,
            'peak_source': 'nominal FP32 SIMT: 148 SMs x 128 lanes x 2 flop x 1965 MHz'}
    simt['frac'] = simt['achieved_tflops'] / FP32_SIMT_TFLOPS
    roofline = {'bound': 'hbm', 'kernel': dominant, 'achieved': achieved, 'peak': peaks['hbm_gbs'], 'unit': 'GB/s',
                'frac': achieved / peaks['hbm_gbs'], 'traffic': profiledTraffic(case, dominant, refine, fluidCount),
                'peak_source': peaks['source'],
                'kernel_ms': kernelMs, 'bytes_per_update': unitBytes, 'step_hbm_frac': unitBytes * fluidCount /
                (totalMs / args.steps / 1e3) / 1e9 / peaks['hbm_gbs']}

    # end to end through the public API with host buffers: push, one step, pull, every step
    e2e = None
    if not args.no_e2e:
        # the device state as it stands (after a split: its count, masses, lengths and flags) in pinned
        # host buffers, pushed whole every step
        current = sums.pullState()
        n, dim = len(current['masses']), case.dimensions
        pinned = {name: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
                  for name, shape in (('positions', (n, dim)), ('velocities', (n, dim)), ('densities', (n,)),
                                      ('masses', (n,)), ('pressures', (n,)), ('accelerations', (n, dim)),
                                      ('lengths', (n,)))}
        flags = torch.empty(n, dtype=torch.bool, pin_memory=True).numpy()
        host = type(state)(pinned['positions'], pinned['velocities'], pinned['accelerations'], pinned['densities'],
                           pinned['pressures'], pinned['masses'], flags)
        for name in ('positions', 'velocities', 'densities', 'masses', 'pressures', 'accelerations'):
            getattr(host, name)[:] = current[name]
        host.isFluid[:] = current['isFluid']
        if refine:
            pinned['lengths'][:] = current['lengths']
            host.lengths = pinned['lengths']
        del current
        bytesIn = n * (dim * 8 * 2 + 8 + 8 + 1 + (8 if refine else 0))
        bytesOut = n * (dim * 8 * 2 + 8 + 8 + dim * 8)
        e2eSteps = max(5, min(args.steps, 20))
        torch.cuda.synchronize()
        begin = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        clockT, clockS, clockDt = t, s, dt
        wall = time.perf_counter()
        begin.record(stream)
        for k in range(e2eSteps):
            sums.push(host)
            clockT, clockS, clockDt = sums.advance(clockT, clockS, math.inf, clockS + 1, h, cfl, maxdt, 0, clockDt)
            sums.pull(host)
        end.record(stream)
        end.synchronize()
        e2eMs = max(begin.elapsed_time(end), 0.0)
        wallMs = (time.perf_counter() - wall) * 1e3
        e2eMs = replicas.maxOverRanks(max(e2eMs, wallMs), ranks)
        e2e = {'value': world * fluidCount * e2eSteps / (e2eMs / 1e3), 'unit': METRIC,
               'h2d_bytes_per_step': bytesIn, 'd2h_bytes_per_step': bytesOut, 'steps': e2eSteps,
               'ms_per_step': e2eMs / e2eSteps}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpuBaseline(case, refine)

    if rank == 0:
        line = {'metric': METRIC, 'value': value, 'unit': METRIC, 'n_gpus': world, 'steps': args.steps,
                'warmup': args.warmup, 'ms_per_step': totalMs / args.steps, 'higher_is_better': True,
                'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32 sums, f64 state', 'data': 'synthetic',
                'config': dict(config(case), parallelism=f'replicas{world}' if world > 1 else 'single',
                               crest_zone_split=refined, fluid_particles_after_split=fluidCount,
                               **sweepConfig(sums, not args.no_table, args.threads or 4)),
                'clocks': clocks, 'e2e': e2e, 'gpu_launches': launchesPerStep * args.steps,
                'roofline': roofline, 'pair_flops': simt, 'stages_ms': stages, 'cpu_baseline': cpu,
                'simulated_time_s': t}
        print(json.dumps(line), flush=True)
    replicas.finalize(ranks)


if __name__ == '__main__':
    main()
