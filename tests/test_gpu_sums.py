"""Each CUDA sum against the reference's float64 array formulation and the float64 oracle.

The clouds and the expected sums are the reference's own (tests/golden/make_golden.py runs
src/pysurf/sphSolver.py on the clouds of tests/testSphGpu.py:32-63).  Tolerances are the
reference's for its float32 device (tests/testSphGpu.py:79-404): 1e-5 of the largest value for
every sum, 2e-5 for the velocity gradients and correction matrices, 2e-4 for the density
gradients.  Neighbour rows and cell keys must match bit for bit.
"""
import numpy as np
import pytest

from conftest import golden, goldenTags
from oracle import oracle

pytestmark = pytest.mark.gpu

CLOUDS = goldenTags('clouds.npz')
rho0, c0, alpha, epsilon = 1000.0, 20.0, 0.1, 0.5


def pairSums(c, precision='float64', **switches):
    from pysurf_b200.sphGpu import PairSums
    x = c['positions']
    kernelType = 'wendlandC2' if int(c['kernel']) == 1 else 'cubicSpline'
    s = PairSums(x.shape[1], float(c['h']), x.min(axis=0), x.max(axis=0), float(c['period']), precision, 'cuda:0',
                 kernelType)
    s.update(x, c['masses'], c['isFluid'])
    return s


def close(result, expected, scale=1e-5):
    tolerance = scale * np.abs(expected).max()
    error = np.abs(result - expected).max()
    assert error <= tolerance, f'error {error:.3e} > {tolerance:.3e}'


@pytest.mark.parametrize('tag', CLOUDS)
def test_accelerations(tag):
    c = golden('clouds.npz', tag)
    dim = c['positions'].shape[1]
    g = np.zeros(dim)
    g[-1] = -9.81
    s = pairSums(c)
    close(s.pairAccelerations(c['velocities'], c['densities'], c['pressures'], c0, alpha, 0.3, g), c['accelerations'])


@pytest.mark.parametrize('tag', CLOUDS)
def test_limited_accelerations_and_velocity_gradients(tag):
    c = golden('clouds.npz', tag)
    dim = c['positions'].shape[1]
    g = np.zeros(dim)
    g[-1] = -9.81
    s = pairSums(c)
    s.setViscosityLimiter(True)
    close(s.velocityGradients(c['strained'], c['densities']), c['velocityGradients'], 2e-5)
    close(s.pairAccelerations(c['strained'], c['densities'], c['pressures'], c0, alpha, 0.3, g),
          c['limitedAccelerations'])


@pytest.mark.parametrize('tag', CLOUDS)
def test_continuity_plain_and_corrected(tag):
    c = golden('clouds.npz', tag)
    s = pairSums(c)
    close(s.continuityRate(c['velocities']), c['continuity'])
    s.setContinuityCorrection(True)
    L = s.correctionMatrices(c['densities'])
    # the cloud's edges hold particles the correction leaves out; float32 must agree on which
    fluid = c['isFluid']
    dim = c['positions'].shape[1]
    assert np.sum(np.all(np.isclose(c['corrections'], np.eye(dim)), axis=(1, 2)) & fluid) > 0
    close(L, c['corrections'], 2e-5)
    close(s.continuityRate(c['velocities'], c['densities']), c['correctedContinuity'])


@pytest.mark.parametrize('tag', CLOUDS)
@pytest.mark.parametrize('mode', ['molteni', 'hydrostatic', 'antuono'])
def test_diffusive_continuity(tag, mode):
    c = golden('clouds.npz', tag)
    s = pairSums(c)
    s.setDiffusion(mode, 0.1, c0, rho0, 9.81)
    if mode == 'antuono':
        close(s.densityGradients(c['densities']), c['densityGradients'], 2e-4)
    close(s.continuityRate(c['velocities'], c['densities']), c[f'diffusive_{mode}'])


@pytest.mark.parametrize('tag', CLOUDS)
def test_wall_pressure_xsph_shepard(tag):
    c = golden('clouds.npz', tag)
    dim = c['positions'].shape[1]
    g = np.zeros(dim)
    g[-1] = -9.81
    s = pairSums(c)
    close(s.wallPressure(c['densities'], c['pressures'], g, rho0, c0), c['wallPressure'])
    fluid = c['isFluid']
    xs = s.xsphVelocity(c['velocities'], c['densities'], epsilon)
    close(xs[fluid], c['xsph'][fluid])
    assert np.allclose(xs[~fluid], c['velocities'][~fluid], atol=1e-6)
    assert np.allclose(s.shepardDensity(c['densities']), c['shepard'], rtol=2e-6, atol=0.0)


@pytest.mark.parametrize('tag', CLOUDS)
def test_sums_match_the_oracle(tag):
    # the same sums against the float64 oracle, for a mixed-length cloud too (h_ij = (h_i + h_j) / 2)
    c = golden('clouds.npz', tag)
    dim = c['positions'].shape[1]
    rng = np.random.default_rng(17)
    lengths = float(c['h']) * rng.choice([1.0, 0.5], size=len(c['masses']))
    kernelType = 'wendlandC2' if int(c['kernel']) == 1 else 'cubicSpline'
    o = oracle.System(c['positions'], c['masses'], c['isFluid'], lengths, kernelType, float(c['period']))
    from pysurf_b200.sphGpu import PairSums
    x = c['positions']
    s = PairSums(dim, float(c['h']), x.min(axis=0), x.max(axis=0), float(c['period']), device='cuda:0',
                 kernelType=kernelType)
    s.update(x, c['masses'], c['isFluid'], lengths)
    g = np.zeros(dim)
    g[-1] = -9.81
    close(s.pairAccelerations(c['velocities'], c['densities'], c['pressures'], c0, alpha, 0.3, g),
          o.pairAccelerations(c['velocities'], c['densities'], c['pressures'], c0, alpha, 0.3, g))
    s.setDiffusion('hydrostatic', 0.1, c0, rho0, 9.81)
    s.setContinuityCorrection(True)
    L = o.correctionMatrices(c['densities'])
    close(s.continuityRate(c['velocities'], c['densities']),
          o.continuityRate(c['velocities'], c['densities'], 'hydrostatic', 0.1, c0, rho0, 9.81, corrections=L))


@pytest.mark.parametrize('tag', CLOUDS)
def test_neighbour_rows_are_the_references_bit_for_bit(tag):
    c = golden('clouds.npz', tag)
    s = pairSums(c)
    offsets, neighbors = s.neighborList(2.0 * float(c['h']))
    assert np.array_equal(np.diff(offsets), np.diff(c['offsets']))
    for i in range(len(offsets) - 1):
        mine = np.sort(neighbors[offsets[i]:offsets[i + 1]])
        theirs = np.sort(c['neighbors'][c['offsets'][i]:c['offsets'][i + 1]])
        assert np.array_equal(mine, theirs), i


def test_cell_keys_are_the_references_bit_for_bit():
    from pysurf_b200.sphGpu import cellOrderKey
    g = np.load('tests/golden/cellkeys.npz')
    assert list(cellOrderKey(g['known3'], 1.0, (4, 3, 2))) == [0, 1, 4, 12, 0, 3]
    assert list(cellOrderKey(g['known2'], 1.0, (4, 3, 1))) == [0, 1, 4]
    assert np.array_equal(cellOrderKey(g['random3'], 0.37, (57, 23, 9)), g['randomKeys3'])
    assert np.array_equal(cellOrderKey(g['random2'], 0.09375, (700, 40, 1)), g['randomKeys2'])


def test_float32_separations_lose_digits_far_from_the_origin():
    # tests/testSphGpu.py:390-404: 25 m out, the point + remainder split keeps the sums to float32
    # rounding of the terms; the float32 points alone do not
    c = golden('clouds.npz', '3d_o_cubicSpline')
    errors = {}
    for precision in ('float64', 'float32'):
        result = pairSums(c, precision).continuityRate(c['velocities'])
        errors[precision] = float(np.abs(result - c['continuity']).max() / np.abs(c['continuity']).max())
    assert errors['float64'] < 1e-5
    assert errors['float32'] > 3.0 * errors['float64']


def test_cells_per_support_changes_nothing_but_the_walk():
    c = golden('clouds.npz', '3d_p_wendlandC2')
    results = []
    for cells in (1, 2, 3):
        s = pairSums(c)
        s.setCellsPerSupport(cells)
        s.update(c['positions'], c['masses'], c['isFluid'])
        results.append(s.continuityRate(c['velocities']))
    close(results[1], c['continuity'])
    close(results[2], c['continuity'])


def test_a_growing_particle_count():
    # tests/testSphGpu.py:406-415: arrays grow when particles are added
    small, large = golden('clouds.npz', '2d_o_cubicSpline'), golden('clouds.npz', '2d_o_cubicSpline')
    s = pairSums(small)
    n = len(small['masses'])
    keep = slice(0, n // 2)
    s.update(small['positions'][keep], small['masses'][keep], small['isFluid'][keep])
    s.update(large['positions'], large['masses'], large['isFluid'])
    assert np.allclose(s.shepardDensity(large['densities']), large['shepard'], rtol=2e-6)


@pytest.mark.parametrize('dimensions', [2, 3])
def test_bed_enforcement(dimensions):
    # tests/testSphGpu.py:645-677: fluid scattered about a reef, a moving piston, the end walls
    from pysurf_b200.state import BedBoundary, ParticleState, Profile
    from pysurf_b200.sphGpu import PairSums
    e = golden('enforce.npz', f'bed{dimensions}d')
    clearance, side, width, offshore, wallX, piston, endLimit = e['params']
    n = len(e['positions'])
    # the fluid, and one boundary particle of the piston carrying its speed
    positions = np.vstack([e['positions'], np.full((1, dimensions), -5.0)])
    velocities = np.vstack([e['velocities'], np.zeros((1, dimensions))])
    velocities[n, 0] = piston
    fluid = np.concatenate([np.ones(n, dtype=bool), [False]])
    state = ParticleState(positions, velocities, np.zeros_like(positions), np.full(n + 1, 1000.0), np.zeros(n + 1),
                          np.full(n + 1, 1.0), fluid)
    profile = Profile(e['bedX'], e['bedZ'], 1.0)
    boundary = BedBoundary(profile, 4.0 * clearance, 3, wallTop=1.5 if offshore else None,
                           width=width if side else None, endWallTop=1.5 if endLimit < profile.endX else None,
                           periodic=False, wallX=wallX)
    boundary._pistonMask = ~fluid
    s = PairSums(dimensions, 1.3 * 0.05, positions.min(axis=0), positions.max(axis=0), device='cuda:0')
    s.setPhysics(1000.0, 10.0, 0.0, 0.0, np.zeros(dimensions), 0.0, 0.0)
    s.push(state)
    s.setBoundary(boundary, state)
    s.enforceBoundary()
    out = s.pullState()
    moved = np.any(out['positions'][:n] != e['positions'], axis=1)
    assert np.count_nonzero(moved) > 0.2 * n
    assert np.allclose(out['positions'][:n], e['enforcedPositions'], rtol=0.0, atol=1e-12)
    assert np.allclose(out['velocities'][:n], e['enforcedVelocities'], rtol=0.0, atol=1e-12)


def test_height_field_enforcement():
    from pysurf_b200.state import HeightFieldBoundary, HeightTable, ParticleState
    from pysurf_b200.sphGpu import PairSums
    e = golden('enforce.npz', 'field')
    ox, oy, sx, sy, clearance, lowY, highY, offshore, lowX, highX = e['params']
    table = e['table']
    ny, nx = table.shape
    gridX, gridY = ox + sx * np.arange(nx), oy + sy * np.arange(ny)
    assert gridX[1] - gridX[0] == sx and gridY[1] - gridY[0] == sy
    field = HeightTable(gridX, gridY, table,
                        (lowX - clearance, highX + clearance, lowY - clearance, highY + clearance))
    boundary = HeightFieldBoundary(field, 4.0 * clearance, 3, 1.5, bool(offshore), True)
    n = len(e['positions'])
    state = ParticleState(e['positions'].copy(), e['velocities'].copy(), np.zeros((n, 3)), np.full(n, 1000.0),
                          np.zeros(n), np.full(n, 1.0), np.ones(n, dtype=bool))
    s = PairSums(3, 3.0 * 0.125, state.positions.min(axis=0), state.positions.max(axis=0), device='cuda:0')
    s.setPhysics(1000.0, 10.0, 0.0, 0.0, np.zeros(3), 0.0, 0.0)
    s.push(state)
    s.setBoundary(boundary, state)
    s.enforceBoundary()
    out = s.pullState()
    assert np.allclose(out['positions'], e['enforcedPositions'], rtol=0.0, atol=1e-12)
    assert np.allclose(out['velocities'], e['enforcedVelocities'], rtol=0.0, atol=1e-12)


@pytest.mark.parametrize('tag', ['3d_p_wendlandC2', '2d_o_cubicSpline'])
@pytest.mark.parametrize('threads', [1, 2, 4, 8])
@pytest.mark.parametrize('table', [True, False])
def test_every_sweep_form_gives_the_reference_sums(tag, threads, table):
    # the neighbour table on or off, one to eight threads a particle: the same sums to float32 rounding
    c = golden('clouds.npz', tag)
    dim = c['positions'].shape[1]
    g = np.zeros(dim)
    g[-1] = -9.81
    s = pairSums(c)
    s.setSweepOptions(table, threads)
    s.update(c['positions'], c['masses'], c['isFluid'])
    close(s.pairAccelerations(c['velocities'], c['densities'], c['pressures'], c0, alpha, 0.3, g), c['accelerations'])
    s.setViscosityLimiter(True)
    close(s.velocityGradients(c['strained'], c['densities']), c['velocityGradients'], 2e-5)
    close(s.pairAccelerations(c['strained'], c['densities'], c['pressures'], c0, alpha, 0.3, g),
          c['limitedAccelerations'])
    s.setDiffusion('antuono', 0.1, c0, rho0, 9.81)
    close(s.densityGradients(c['densities']), c['densityGradients'], 2e-4)
    close(s.continuityRate(c['velocities'], c['densities']), c['diffusive_antuono'])
    close(s.wallPressure(c['densities'], c['pressures'], g, rho0, c0), c['wallPressure'])
    fluid = c['isFluid']
    close(s.xsphVelocity(c['velocities'], c['densities'], epsilon)[fluid], c['xsph'][fluid])
    assert np.allclose(s.shepardDensity(c['densities']), c['shepard'], rtol=2e-6, atol=0.0)


@pytest.mark.parametrize('tag', CLOUDS)
def test_closure_sums(tag):
    # the delta-LES-SPH closure (src/pysurf/sphSolver.py:1232-1326) under the strained flow: the
    # coefficients, the accelerations with its viscous term, the continuity with its diffusion
    c, k = golden('clouds.npz', tag), golden('closure.npz', tag)
    nu = float(np.load('tests/golden/closure.npz')['viscosity'])
    dim = c['positions'].shape[1]
    g = np.zeros(dim)
    g[-1] = -9.81
    s = pairSums(c)
    s.setClosure(True, c0, rho0, nu)
    s.setDiffusion('hydrostatic', 0.1, c0, rho0, 9.81)
    alphas, deltas = s.closureCoefficients(c['strained'], c['densities'])
    close(alphas, k['alphas'], 2e-4)
    close(deltas, k['deltas'], 2e-4)
    close(s.pairAccelerations(c['strained'], c['densities'], c['pressures'], c0, alpha, 0.3, g), k['accelerations'])
    # the continuity takes the deltas of the last accelerations, as the reference's device does
    close(s.continuityRate(c['strained'], c['densities']), k['continuity'])


SHIFT_CLOUDS = ['2d_cubicSpline', '2d_wendlandC2', '3d_cubicSpline', '3d_wendlandC2']


@pytest.mark.parametrize('tag', SHIFT_CLOUDS)
def test_shifting_displacement(tag):
    # particle shifting (src/pysurf/sphSolver.py:824-1010) on water over a wall layer: the same
    # particles shift, by the reference's shifts, density and velocity changes
    from pysurf_b200.sphGpu import PairSums
    k = golden('shifting.npz', tag)
    x = k['positions']
    kernelType = 'wendlandC2' if int(k['kernel']) == 1 else 'cubicSpline'
    s = PairSums(x.shape[1], float(k['h']), x.min(axis=0), x.max(axis=0), 0.0, 'float64', 'cuda:0', kernelType)
    s.update(x, k['masses'], k['isFluid'])
    h, spacing = float(k['h']), 0.02
    # size CFL Ma (2h)^2 with CFL = c0 dt / h: the fixture's 0.2 x 0.1 x (2h)^2 at c0 20, Ma 0.1
    s.setShifting(True, 0.1, spacing, c0, False)
    dt = 0.2 * h / c0
    shift, densityChange, velocityChange = s.shiftingDisplacement(k['densities'], dt, k['velocities'])
    assert np.array_equal(np.abs(shift).sum(1) > 0, np.abs(k['shift']).sum(1) > 0)
    close(shift, k['shift'])
    close(densityChange, k['densityChange'])
    close(velocityChange, k['velocityChange'])
