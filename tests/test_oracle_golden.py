"""The float64 oracle against golden vectors made by the reference itself (tests/golden/make_golden.py).

These pin the oracle before it is trusted as the CUDA backend's checker: cell keys and neighbour
rows bit-exact, every sum to float64 rounding, enforcement to 1e-12, split exact, and the
device-resident step against the reference's own float64 host steps.
"""
import numpy as np
import pytest

from conftest import golden, goldenTags
from oracle import oracle


def test_cell_keys_known_answer():
    # tests/testSphSolver.py:818-824: x fastest, then y, then z, wrapped onto the grid
    g = np.load('tests/golden/cellkeys.npz')
    assert list(oracle.cellOrderKey(g['known3'], 1.0, (4, 3, 2))) == [0, 1, 4, 12, 0, 3]
    assert list(oracle.cellOrderKey(g['known2'], 1.0, (4, 3, 1))) == [0, 1, 4]
    assert np.array_equal(oracle.cellOrderKey(g['random3'], 0.37, (57, 23, 9)), g['randomKeys3'])
    assert np.array_equal(oracle.cellOrderKey(g['random2'], 0.09375, (700, 40, 1)), g['randomKeys2'])


CLOUDS = goldenTags('clouds.npz')


def system(c):
    kernelType = 'wendlandC2' if int(c['kernel']) == 1 else 'cubicSpline'
    return oracle.System(c['positions'], c['masses'], c['isFluid'], float(c['h']), kernelType, float(c['period']))


def close(result, expected, scale=1e-9):
    return np.allclose(result, expected, rtol=0.0, atol=scale * max(np.abs(expected).max(), 1e-300))


@pytest.mark.parametrize('tag', CLOUDS)
def test_neighbor_rows_match_the_reference_element_for_element(tag):
    c = golden('clouds.npz', tag)
    offsets, neighbors = oracle.neighborList(c['positions'], 2.0 * float(c['h']), float(c['period']))
    assert np.array_equal(offsets, c['offsets'])
    assert np.array_equal(neighbors, c['neighbors'])
    # and the rows hold exactly the cKDTree pair set, each pair from both sides
    assert offsets[-1] == 2 * int(c['pairCount'])


@pytest.mark.parametrize('tag', CLOUDS)
def test_sums_match_the_reference_array_formulation(tag):
    c = golden('clouds.npz', tag)
    s = system(c)
    dim = c['positions'].shape[1]
    g = np.zeros(dim)
    g[-1] = -9.81
    rho0, c0, alpha = 1000.0, 20.0, 0.1
    assert close(s.pairAccelerations(c['velocities'], c['densities'], c['pressures'], c0, alpha, 0.3, g),
                 c['accelerations'])
    G = s.velocityGradients(c['strained'], c['densities'])
    assert close(G, c['velocityGradients'])
    assert close(s.pairAccelerations(c['strained'], c['densities'], c['pressures'], c0, alpha, 0.3, g, G),
                 c['limitedAccelerations'])
    assert close(s.continuityRate(c['velocities']), c['continuity'])
    L = s.correctionMatrices(c['densities'])
    assert close(L, c['corrections'])
    assert close(s.continuityRate(c['velocities'], c['densities'], corrections=L), c['correctedContinuity'])
    for mode in ('molteni', 'hydrostatic'):
        assert close(s.continuityRate(c['velocities'], c['densities'], mode, 0.1, c0, rho0, 9.81),
                     c[f'diffusive_{mode}'])
    gr = s.densityGradients(c['densities'], L)
    assert close(gr, c['densityGradients'])
    assert close(s.continuityRate(c['velocities'], c['densities'], 'antuono', 0.1, c0, rho0, 9.81, gradients=gr),
                 c['diffusive_antuono'])
    p, rho = s.wallPressure(c['densities'], c['pressures'], g, rho0, c0)
    assert close(p, c['wallPressure'])
    assert close(rho, c['wallDensity'], 1e-13)
    assert close(s.xsphVelocity(c['velocities'], c['densities'], 0.5), c['xsph'])
    assert close(s.shepardDensity(c['densities']), c['shepard'], 1e-13)


@pytest.mark.parametrize('dimensions', [2, 3])
def test_bed_enforcement_matches_the_reference(dimensions):
    e = golden('enforce.npz', f'bed{dimensions}d')
    clearance, side, width, offshore, wallX, piston, endLimit = e['params']
    params = oracle.bedParams(e['bedX'], e['bedZ'], clearance, bool(side), width, bool(offshore), wallX, piston,
                              endLimit)
    fluid = np.ones(len(e['positions']), dtype=bool)
    x, v = oracle.enforceBed(e['positions'], e['velocities'], fluid, params)
    assert np.count_nonzero(np.any(x != e['positions'], axis=1)) > 0.2 * len(x)
    assert np.allclose(x, e['enforcedPositions'], rtol=0.0, atol=1e-12)
    assert np.allclose(v, e['enforcedVelocities'], rtol=0.0, atol=1e-12)


def test_height_field_enforcement_matches_the_reference():
    e = golden('enforce.npz', 'field')
    ox, oy, sx, sy, clearance, lowY, highY, offshore, lowX, highX = e['params']
    params = oracle.fieldParams(e['table'], ox, oy, sx, sy, clearance, lowY, highY, bool(offshore), lowX, highX)
    fluid = np.ones(len(e['positions']), dtype=bool)
    x, v = oracle.enforceHeightField(e['positions'], e['velocities'], fluid, params)
    assert np.count_nonzero(np.any(x != e['positions'], axis=1)) > 0.2 * len(x)
    assert np.allclose(x, e['enforcedPositions'], rtol=0.0, atol=1e-12)
    assert np.allclose(v, e['enforcedVelocities'], rtol=0.0, atol=1e-12)


@pytest.mark.parametrize('tag', goldenTags('split.npz'))
def test_split_matches_the_reference(tag):
    s = golden('split.npz', tag)
    ratio = float(tag.split('_')[1])
    state = {k: s[k].copy() for k in ('positions', 'velocities', 'accelerations', 'densities', 'pressures',
                                       'masses', 'isFluid')}
    count = oracle.splitParticles(state, s['mask'], 1000.0, 1.3 * 0.05, ratio)
    assert count == int(s['count'])
    for key in ('positions', 'velocities', 'accelerations', 'densities', 'pressures', 'lengths'):
        assert np.allclose(state[key], s[f'split_{key}'], rtol=1e-15, atol=1e-15), key
    # mass is conserved exactly: m / 2^dim is a power-of-two division
    assert np.array_equal(state['masses'], s['split_masses'])
    assert np.array_equal(state['isFluid'], s['split_isFluid'])
    assert state['masses'].sum() == pytest.approx(s['masses'].sum(), rel=1e-15)


def stepperFor(r, **options):
    (dim, kind, h, rho0, c0, alpha, bf, xsph, floor, mode, delta, wall, tension, corrected, limited, cfl, maxdt,
     interval, period) = r['config']
    modes = ['none', 'molteni', 'hydrostatic', 'antuono']
    boundary = None
    if int(r['boundary_kind']) == 1:
        boundary = ('container', r['boundary_lower'], r['boundary_upper'], bool(r['boundary_openTop']))
    elif int(r['boundary_kind']) == 2:
        clearance, side, width, offshore, wallX, piston, endLimit = r['boundary_params']
        boundary = ('bed', oracle.bedParams(r['boundary_bedX'], r['boundary_bedZ'], clearance, bool(side), width,
                                            bool(offshore), wallX, piston, endLimit))
    elif int(r['boundary_kind']) == 3:
        ox, oy, sx, sy, clearance, lowY, highY, offshore, lowX, highX = r['boundary_params']
        boundary = ('field', oracle.fieldParams(r['boundary_table'], ox, oy, sx, sy, clearance, lowY, highY,
                                                bool(offshore), lowX, highX))
    return oracle.Stepper(int(dim), 'wendlandC2' if int(kind) == 1 else 'cubicSpline', h, rho0, c0, alpha,
                          r['gravity'], bf, xsph, floor, modes[int(mode)], delta, bool(wall), bool(tension),
                          bool(corrected), bool(limited), cfl, maxdt, period, int(interval), boundary, **options)


@pytest.mark.parametrize('tag', goldenTags('runs.npz'))
def test_device_step_follows_the_reference_host_steps(tag):
    r = golden('runs.npz', tag)
    stepper = stepperFor(r)
    state = {k: r[k].copy() for k in ('positions', 'velocities', 'densities', 'masses', 'isFluid')}
    dts = [stepper(state) for _ in range(int(r['steps']))]
    assert np.allclose(dts, r['dts'], rtol=1e-10, atol=0.0)
    assert np.allclose(state['positions'], r['finalPositions'], rtol=0.0, atol=1e-11)
    assert np.allclose(state['velocities'], r['finalVelocities'], rtol=0.0, atol=1e-8)
    assert np.allclose(state['densities'], r['finalDensities'], rtol=1e-11, atol=0.0)
    fluid = r['isFluid']
    assert np.allclose(state['accelerations'][fluid], r['finalAccelerations'][fluid], rtol=0.0,
                       atol=1e-8 * np.abs(r['finalAccelerations']).max())


@pytest.mark.parametrize('tag', goldenTags('runs3d.npz'))
def test_device_step_follows_the_reference_host_steps_in_3d(tag):
    # the reference's BreakingWave3D tank over a ridge (height-field bed, walls six layers deep), its
    # numpy solver's host steps, whole and after a crest split into daughters of h / 2
    r = golden('runs3d.npz', tag)
    stepper = stepperFor(r)
    state = {k: r[k].copy() for k in ('positions', 'velocities', 'densities', 'masses', 'isFluid', 'lengths')}
    dts = [stepper(state) for _ in range(int(r['steps']))]
    assert np.allclose(dts, r['dts'], rtol=1e-10, atol=0.0)
    assert np.allclose(state['positions'], r['finalPositions'], rtol=0.0, atol=1e-11)
    assert np.allclose(state['velocities'], r['finalVelocities'], rtol=0.0, atol=1e-8)
    assert np.allclose(state['densities'], r['finalDensities'], rtol=1e-11, atol=0.0)


def closureGolden(tag):
    return golden('closure.npz', tag)


@pytest.mark.parametrize('tag', CLOUDS)
def test_closure_sums_match_the_reference(tag):
    # src/pysurf/sphSolver.py:1232-1326: coefficients from the strained flow's gradients, the
    # delta-LES-SPH viscous term on every fluid pair, the diffusion at the pairs' harmonic-mean delta
    c, k = golden('clouds.npz', tag), closureGolden(tag)
    nu = float(np.load('tests/golden/closure.npz')['viscosity'])
    s = system(c)
    dim = c['positions'].shape[1]
    g = np.zeros(dim)
    g[-1] = -9.81
    rho0, c0, alpha = 1000.0, 20.0, 0.1
    G = s.velocityGradients(c['strained'], c['densities'])
    alphas, deltas = s.closureCoefficients(G, c0)
    assert close(alphas, k['alphas']) and close(deltas, k['deltas'])
    assert close(s.pairAccelerations(c['strained'], c['densities'], c['pressures'], c0, alpha, 0.3, g, G, limited=False,
                                     closure=(alphas, nu, rho0)), k['accelerations'])
    assert close(s.continuityRate(c['strained'], c['densities'], 'hydrostatic', 0.1, c0, rho0, 9.81, deltas=deltas),
                 k['continuity'])


def test_closure_step_follows_the_reference_host_steps():
    r = closureGolden('closure')
    base = stepperFor(r)
    sp = base.params
    stepper = oracle.Stepper(int(sp.dim), 'wendlandC2' if sp.kind == 1 else 'cubicSpline', sp.hMax, sp.rho0, sp.c0,
                             sp.alpha, r['gravity'], sp.boundaryFactor, sp.xsphEpsilon, sp.densityFloor,
                             ['none', 'molteni', 'hydrostatic', 'antuono'][sp.diffusion], sp.delta,
                             bool(sp.wallExtrapolated), bool(sp.tension), bool(sp.corrected), bool(sp.limited),
                             sp.cfl, sp.maxTimeStep, sp.period, base.filterInterval,
                             ('container', r['boundary_lower'], r['boundary_upper'], bool(r['boundary_openTop'])),
                             closure=True, viscosity=float(np.load('tests/golden/closure.npz')['viscosity']))
    state = {k: r[k].copy() for k in ('positions', 'velocities', 'densities', 'masses', 'isFluid')}
    dts = [stepper(state) for _ in range(int(r['steps']))]
    assert np.allclose(dts, r['dts'], rtol=1e-10, atol=0.0)
    assert np.allclose(state['positions'], r['finalPositions'], rtol=0.0, atol=1e-11)
    assert np.allclose(state['velocities'], r['finalVelocities'], rtol=0.0, atol=1e-8)
    assert np.allclose(state['densities'], r['finalDensities'], rtol=1e-11, atol=0.0)


SHIFT_CLOUDS = ['2d_cubicSpline', '2d_wendlandC2', '3d_cubicSpline', '3d_wendlandC2']


@pytest.mark.parametrize('tag', SHIFT_CLOUDS)
def test_shifting_matches_the_reference(tag):
    # src/pysurf/sphSolver.py:824-1010 on water over a wall layer: fields, shift, density and velocity changes
    k = golden('shifting.npz', tag)
    kernelType = 'wendlandC2' if int(k['kernel']) == 1 else 'cubicSpline'
    s = oracle.System(k['positions'], k['masses'], k['isFluid'], float(k['h']), kernelType, 0.0)
    fluid = k['isFluid']
    fields = s.shiftingFields(k['densities'], float(k['spacingKernel']))
    for got, name in zip(fields, ('gradient', 'plain', 'divergence', 'densityGradient')):
        assert close(got[fluid], k[name][fluid]), name
    dim = k['positions'].shape[1]
    shift, drho, dv = s.shift(k['densities'], k['velocities'], fields, float(k['size']), {2: 1.5, 3: 2.4}[dim],
                              0.4 if kernelType == 'wendlandC2' else 0.3)
    assert np.array_equal(np.abs(shift).sum(1) > 0, np.abs(k['shift']).sum(1) > 0)
    assert close(shift, k['shift']) and close(drho, k['densityChange']) and close(dv, k['velocityChange'])


def test_shifting_step_follows_the_reference_host_steps():
    r = golden('shifting.npz', 'shifting')
    base = stepperFor(r)
    sp = base.params
    stepper = oracle.Stepper(int(sp.dim), 'wendlandC2' if sp.kind == 1 else 'cubicSpline', sp.hMax, sp.rho0, sp.c0,
                             sp.alpha, r['gravity'], sp.boundaryFactor, sp.xsphEpsilon, sp.densityFloor,
                             ['none', 'molteni', 'hydrostatic', 'antuono'][sp.diffusion], sp.delta,
                             bool(sp.wallExtrapolated), bool(sp.tension), bool(sp.corrected), bool(sp.limited),
                             sp.cfl, sp.maxTimeStep, sp.period, base.filterInterval,
                             ('container', r['boundary_lower'], r['boundary_upper'], bool(r['boundary_openTop'])),
                             shifting=True, shiftingMach=float(r['mach']), spacing=float(r['spacing']))
    state = {k: r[k].copy() for k in ('positions', 'velocities', 'densities', 'masses', 'isFluid')}
    dts = [stepper(state) for _ in range(int(r['steps']))]
    assert np.allclose(dts, r['dts'], rtol=1e-10, atol=0.0)
    assert np.allclose(state['positions'], r['finalPositions'], rtol=0.0, atol=1e-11)
    assert np.allclose(state['velocities'], r['finalVelocities'], rtol=0.0, atol=1e-8)
    assert np.allclose(state['densities'], r['finalDensities'], rtol=1e-11, atol=0.0)
