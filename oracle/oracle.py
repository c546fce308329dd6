"""FP64 CPU oracle for pySurf's delta-SPH step -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this module; the
product (``pysurf_b200``) never does.  It wraps ``sph_oracle.c`` (a float64 restatement of the
reference's sums in gather form, citations there) and adds the two pieces of bookkeeping that
are plainer in numpy:

    splitParticles      src/pysurf/sphRefinement.py:136-190
    crestZone           the device's crest zone (sph_split_crest_zone), for the CPU baseline's sample
    solitaryWaveBeach   (set-up only) see pysurf_b200.cases

Every function takes and returns numpy float64 arrays shaped as the reference's array
formulation does: vectors (N, dim), matrices (N, dim, dim), scalars (N,).
"""
from __future__ import annotations

import ctypes as C
import itertools

import numpy as np

from oracle.build import build

_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags='C_CONTIGUOUS')
_ip64 = np.ctypeslib.ndpointer(dtype=np.int64, flags='C_CONTIGUOUS')
_ip32 = np.ctypeslib.ndpointer(dtype=np.int32, flags='C_CONTIGUOUS')
_u8 = np.ctypeslib.ndpointer(dtype=np.uint8, flags='C_CONTIGUOUS')
_vp = C.c_void_p


class BedParams(C.Structure):
    _fields_ = [('bedX', _vp), ('bedZ', _vp), ('count', C.c_long), ('clearance', C.c_double),
                ('sideWalls', C.c_int), ('width', C.c_double), ('offshoreWall', C.c_int),
                ('wallX', C.c_double), ('pistonSpeed', C.c_double), ('endLimit', C.c_double)]


class FieldParams(C.Structure):
    _fields_ = [('table', _vp), ('nx', C.c_long), ('ny', C.c_long), ('originX', C.c_double),
                ('originY', C.c_double), ('stepX', C.c_double), ('stepY', C.c_double),
                ('clearance', C.c_double), ('lowY', C.c_double), ('highY', C.c_double),
                ('offshoreWall', C.c_int), ('lowX', C.c_double), ('highX', C.c_double)]


class StepParams(C.Structure):
    _fields_ = [('dim', C.c_int), ('kind', C.c_int), ('period', C.c_double), ('hMax', C.c_double),
                ('hMin', C.c_double), ('rho0', C.c_double), ('c0', C.c_double), ('alpha', C.c_double),
                ('boundaryFactor', C.c_double), ('g', C.c_double * 3), ('xsphEpsilon', C.c_double),
                ('densityFloor', C.c_double), ('diffusion', C.c_int), ('delta', C.c_double),
                ('wallExtrapolated', C.c_int), ('tension', C.c_int), ('corrected', C.c_int),
                ('limited', C.c_int), ('cfl', C.c_double), ('maxTimeStep', C.c_double),
                ('filterDensity', C.c_int), ('boundaryKind', C.c_int), ('lower', C.c_double * 3),
                ('upper', C.c_double * 3), ('openTop', C.c_int), ('bed', BedParams), ('field', FieldParams),
                ('closure', C.c_int), ('viscosity', C.c_double), ('shifting', C.c_int), ('shiftLocal', C.c_int),
                ('shiftMach', C.c_double), ('spacingKernel', C.c_double), ('shiftThreshold', C.c_double),
                ('lopsidedness', C.c_double), ('energy', _vp)]


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        L = _lib
        sysargs = [C.c_int, C.c_int, C.c_double, _dp, _dp, _u8, _dp, _ip64, _ip32]
        L.or_cell_order_key.argtypes = [_dp, C.c_long, C.c_int, C.c_double, _ip64, _ip64]
        L.or_neighbor_list.argtypes = [_dp, C.c_long, C.c_int, C.c_double, C.c_double, _ip64, _vp]
        L.or_neighbor_list.restype = C.c_long
        L.or_equation_of_state.argtypes = [C.c_long, _dp, _u8, C.c_double, C.c_double, C.c_int, _dp]
        L.orx_wall_pressure.argtypes = sysargs + [C.c_long, _dp, _dp, _dp, C.c_double, C.c_double, _dp, _dp]
        L.orx_velocity_gradients.argtypes = sysargs + [C.c_long, _dp, _dp, _dp]
        L.orx_correction_matrices.argtypes = sysargs + [C.c_long, _dp, _dp]
        L.orx_density_gradients.argtypes = sysargs + [C.c_long, _dp, _dp, _dp]
        L.orx_accelerations.argtypes = sysargs + [C.c_long, _dp, _dp, _dp, _vp, C.c_double, C.c_double,
                                                  C.c_double, _dp, C.c_int, C.c_int, C.c_double, C.c_double, _vp,
                                                  _dp]
        L.orx_continuity.argtypes = sysargs + [C.c_long, _dp, _dp, _vp, _vp, C.c_int, C.c_double, C.c_double,
                                               C.c_double, C.c_double, C.c_int, C.c_int, _vp, _dp]
        L.orx_closure_coefficients.argtypes = sysargs + [C.c_long, _dp, C.c_double, _dp, _dp]
        L.orx_kernel_value.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double]
        L.orx_kernel_value.restype = C.c_double
        L.orx_shifting_fields.argtypes = sysargs + [C.c_long, _dp, C.c_double, _dp, _dp, _dp, _dp]
        L.orx_shift.argtypes = sysargs + [C.c_long, _dp, _dp, _dp, _dp, _dp, _dp, _dp, C.c_double, C.c_double, _dp,
                                          _dp, _dp]
        L.orx_xsph.argtypes = sysargs + [C.c_long, _dp, _dp, C.c_double, _dp]
        L.orx_shepard.argtypes = sysargs + [C.c_long, _dp, _dp]
        L.or_step.argtypes = [C.POINTER(StepParams), C.c_long, _dp, _dp, _dp, _dp, _dp, _u8, _dp, _dp]
        L.or_step.restype = C.c_double
        L.or_enforce_container.argtypes = [C.c_long, C.c_int, _dp, _dp, _u8, _dp, _dp, C.c_int]
        L.or_enforce_bed.argtypes = [C.c_long, C.c_int, _dp, _dp, _u8, C.POINTER(BedParams)]
        L.or_enforce_heightfield.argtypes = [C.c_long, _dp, _dp, _u8, C.POINTER(FieldParams)]
        L.orx_step_size.restype = C.c_long
        L.or_elastic_energy.argtypes = [C.c_long, _dp, C.c_double, C.c_double, C.c_int, _dp]
        L.or_elastic_slope.argtypes = [C.c_long, _dp, _dp, C.c_double, C.c_double, C.c_int, _dp]
        L.or_fluid_energy.argtypes = [C.c_long, C.c_int, _dp, _dp, _dp, _dp, _u8, _dp, C.c_double, C.c_double,
                                      C.c_int, _dp]
        assert L.orx_step_size() == C.sizeof(StepParams), 'StepParams layout mismatch'
    return _lib


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _u8a(a):
    return np.ascontiguousarray(np.asarray(a).astype(np.uint8))


def cellOrderKey(positions, cellWidth, shape):
    """src/pysurf/sphSolver.py:1379-1408."""
    x = _f64(positions)
    keys = np.empty(len(x), dtype=np.int64)
    shp = np.array(list(shape) + [1] * (3 - len(shape)), dtype=np.int64)
    lib().or_cell_order_key(x, len(x), x.shape[1], float(cellWidth), shp, keys)
    return keys


def neighborList(positions, radius, period=0.0):
    """src/pysurf/sphCompiled.py:133-234: (offsets int64 (N+1,), neighbors int32), reference order."""
    x = _f64(positions)
    n, dim = x.shape
    offsets = np.zeros(n + 1, dtype=np.int64)
    total = lib().or_neighbor_list(x, n, dim, float(radius), float(period or 0.0), offsets, None)
    neighbors = np.empty(max(total, 1), dtype=np.int32)
    lib().or_neighbor_list(x, n, dim, float(radius), float(period or 0.0), offsets,
                           neighbors.ctypes.data_as(C.c_void_p))
    return offsets, neighbors[:total]


class System:
    """A particle set with its neighbour rows at radius 2 max(h), for the sums."""

    def __init__(self, positions, masses, isFluid, h, kernelType='cubicSpline', period=0.0):
        self.x = _f64(positions)
        self.n, self.dim = self.x.shape
        self.m = _f64(np.broadcast_to(masses, (self.n,)))
        self.fluid = _u8a(isFluid)
        self.h = _f64(np.broadcast_to(h, (self.n,)))
        self.kind = 1 if kernelType == 'wendlandC2' else 0
        self.period = float(period or 0.0)
        self.offsets, self.neighbors = neighborList(self.x, 2.0 * float(self.h.max()), self.period)
        if len(self.neighbors) == 0:
            self.neighbors = np.zeros(1, dtype=np.int32)

    def _args(self):
        return (self.dim, self.kind, self.period, self.x, self.h, self.fluid, self.m, self.offsets, self.neighbors)

    def _vec(self, a):
        return _f64(a).reshape(self.n, self.dim)

    def wallPressure(self, densities, pressures, gravity, rho0, c0):
        """src/pysurf/sphSolver.py:1045-1106 with the boundary's Tait density (sphGpu.py:804-854)."""
        p, rho = np.empty(self.n), np.empty(self.n)
        lib().orx_wall_pressure(*self._args(), self.n, _f64(densities), _f64(pressures),
                                _f64(np.resize(gravity, 3)), rho0, c0, p, rho)
        return p, rho

    def velocityGradients(self, velocities, densities):
        out = np.empty((self.n, self.dim, self.dim))
        lib().orx_velocity_gradients(*self._args(), self.n, self._vec(velocities), _f64(densities), out)
        return out

    def correctionMatrices(self, densities):
        out = np.empty((self.n, self.dim, self.dim))
        lib().orx_correction_matrices(*self._args(), self.n, _f64(densities), out)
        return out

    def densityGradients(self, densities, corrections=None):
        L = self.correctionMatrices(densities) if corrections is None else _f64(corrections)
        out = np.empty((self.n, self.dim))
        lib().orx_density_gradients(*self._args(), self.n, _f64(densities), L, out)
        return out

    def pairAccelerations(self, velocities, densities, pressures, c0, alpha, boundaryFactor, gravity,
                          gradients=None, limited=None, closure=None):
        """limited: the limiter (by default on when `gradients` are given); closure: None, or
        (alphas, viscosity, rho0) for the delta-LES-SPH term (src/pysurf/sphSolver.py:1283-1326)."""
        out = np.empty((self.n, self.dim))
        G = None if gradients is None else _f64(gradients)
        limited = G is not None if limited is None else bool(limited)
        alphas, waterTerm, rho0 = None, 0.0, 1000.0
        if closure is not None:
            alphas = _f64(closure[0])
            waterTerm = 2.0 * (self.dim + 2) * float(closure[1]) / c0
            rho0 = float(closure[2])
        lib().orx_accelerations(*self._args(), self.n, self._vec(velocities), _f64(densities), _f64(pressures),
                                None if G is None else G.ctypes.data_as(C.c_void_p), c0, alpha, boundaryFactor,
                                _f64(np.resize(gravity, 3)), int(limited), int(closure is not None), waterTerm, rho0,
                                None if alphas is None else alphas.ctypes.data_as(C.c_void_p), out)
        return out

    def shiftingFields(self, densities, spacingKernel):
        """src/pysurf/sphSolver.py:824-887: grad C, grad C0, div r and grad rho (fluid rows)."""
        grad, plain, rg = (np.empty((self.n, self.dim)) for _ in range(3))
        div = np.empty(self.n)
        lib().orx_shifting_fields(*self._args(), self.n, _f64(densities), float(spacingKernel), grad, plain, div, rg)
        return grad, plain, div, rg

    def shift(self, densities, velocities, fields, size, threshold, lopsidedness):
        """src/pysurf/sphSolver.py:889-1010: the shifts, density and velocity changes."""
        grad, plain, div, rg = (_f64(f) for f in fields)
        shift, dv = np.empty((self.n, self.dim)), np.empty((self.n, self.dim))
        drho = np.empty(self.n)
        lib().orx_shift(*self._args(), self.n, _f64(densities), self._vec(velocities), grad, plain, div, rg,
                        _f64(np.broadcast_to(size, (self.n,))), float(threshold), float(lopsidedness), shift, drho, dv)
        return shift, drho, dv

    def closureCoefficients(self, gradients, c0):
        """src/pysurf/sphSolver.py:1232-1274: each particle's alpha_i and delta_i."""
        alphas, deltas = np.empty(self.n), np.empty(self.n)
        lib().orx_closure_coefficients(*self._args(), self.n, _f64(gradients), c0, alphas, deltas)
        return alphas, deltas

    def continuityRate(self, velocities, densities=None, mode='none', delta=0.1, c0=20.0, rho0=1000.0,
                       gravity=9.81, corrections=None, gradients=None, deltas=None):
        """deltas: each particle's closure delta_i, whose pair harmonic mean replaces `delta`."""
        modes = {'none': 0, 'molteni': 1, 'hydrostatic': 2, 'antuono': 3}
        rho = _f64(densities if densities is not None else np.full(self.n, rho0))
        L = None if corrections is None else _f64(corrections)
        gr = None if gradients is None else _f64(gradients)
        if modes[mode] == 3 and gr is None:
            gr = self.densityGradients(rho)
        out = np.empty(self.n)
        lib().orx_continuity(*self._args(), self.n, self._vec(velocities), rho,
                             None if L is None else L.ctypes.data_as(C.c_void_p),
                             None if gr is None else gr.ctypes.data_as(C.c_void_p), modes[mode], delta, c0, rho0,
                             gravity, int(L is not None), int(deltas is not None),
                             None if deltas is None else _f64(deltas).ctypes.data_as(C.c_void_p), out)
        return out

    def xsphVelocity(self, velocities, densities, epsilon):
        out = np.empty((self.n, self.dim))
        lib().orx_xsph(*self._args(), self.n, self._vec(velocities), _f64(densities), epsilon, out)
        return out

    def shepardDensity(self, densities):
        out = np.empty(self.n)
        lib().orx_shepard(*self._args(), self.n, _f64(densities), out)
        return out


def equationOfState(densities, isFluid, rho0, c0, tension=False):
    rho = _f64(densities)
    out = np.empty(len(rho))
    lib().or_equation_of_state(len(rho), rho, _u8a(isFluid), rho0, c0, int(tension), out)
    return out


def bedParams(bedX, bedZ, clearance, sideWalls=False, width=0.0, offshoreWall=False, wallX=0.0, pistonSpeed=0.0,
              endLimit=np.inf):
    bx, bz = _f64(bedX), _f64(bedZ)
    p = BedParams(bx.ctypes.data, bz.ctypes.data, len(bx), clearance, int(sideWalls), width, int(offshoreWall),
                  wallX, pistonSpeed, endLimit)
    p._keep = (bx, bz)
    return p


def fieldParams(table, originX, originY, stepX, stepY, clearance, lowY, highY, offshoreWall, lowX, highX):
    t = _f64(table)
    p = FieldParams(t.ctypes.data, t.shape[1], t.shape[0], originX, originY, stepX, stepY, clearance, lowY, highY,
                    int(offshoreWall), lowX, highX)
    p._keep = (t,)
    return p


def enforceContainer(positions, velocities, isFluid, lower, upper, openTop=True):
    x, v = _f64(positions).copy(), _f64(velocities).copy()
    lib().or_enforce_container(len(x), x.shape[1], x, v, _u8a(isFluid), _f64(lower), _f64(upper), int(openTop))
    return x, v


def enforceBed(positions, velocities, isFluid, params):
    x, v = _f64(positions).copy(), _f64(velocities).copy()
    lib().or_enforce_bed(len(x), x.shape[1], x, v, _u8a(isFluid), C.byref(params))
    return x, v


def enforceHeightField(positions, velocities, isFluid, params):
    x, v = _f64(positions).copy(), _f64(velocities).copy()
    lib().or_enforce_heightfield(len(x), x, v, _u8a(isFluid), C.byref(params))
    return x, v


# The energy budget's terms the steps keep, in the order of src/pysurf/sphEnergy.py:92-98 (deviceTerms)
ENERGY_TERMS = ('pressureFluid', 'viscosityFluid', 'pressureWall', 'viscosityWall', 'gravityWork', 'continuityFluid',
                'continuityWall', 'correction', 'diffusion', 'floor', 'drift', 'clamp', 'shifting', 'filter')


def elasticEnergy(densities, rho0, c0, tension=False):
    """src/pysurf/sphEnergy.py:100-139: the Tait elastic energy per unit mass [J/kg]."""
    rho = _f64(np.atleast_1d(densities))
    out = np.empty_like(rho)
    lib().or_elastic_energy(len(rho), rho, rho0, c0, int(tension), out)
    return out


def elasticSlope(before, after, rho0, c0, tension=False):
    """src/pysurf/sphEnergy.py:141-160: the secant slope of e, or p / rho^2 for a tiny change."""
    a, b = np.broadcast_arrays(_f64(np.atleast_1d(before)), _f64(np.atleast_1d(after)))
    out = np.empty(a.shape)
    lib().or_elastic_slope(len(out), _f64(a), _f64(b), rho0, c0, int(tension), out)
    return out


def fluidEnergy(state, gravity, rho0, c0, tension=False):
    """The fluid's kinetic, potential and elastic energy [J] (per unit depth in 2D)."""
    x = _f64(state['positions'])
    n, dim = x.shape
    out = np.empty(3)
    lib().or_fluid_energy(n, dim, x, _f64(state['velocities']), _f64(state['densities']), _f64(state['masses']),
                          _u8a(state['isFluid']), _f64(np.resize(gravity, 3)), rho0, c0, int(tension), out)
    return out


class Stepper:
    """The device-resident step of src/pysurf/sphGpu.py:2237-2315 in float64, one call per step."""

    diffusionModes = {'none': 0, 'molteni': 1, 'hydrostatic': 2, 'antuono': 3}

    def __init__(self, dim, kernelType, hMax, rho0, c0, alpha, gravity, boundaryFactor=0.0, xsphEpsilon=0.0,
                 densityFloor=0.0, diffusion='none', delta=0.1, wallExtrapolated=False, tension=False,
                 corrected=False, limited=False, cfl=0.25, maxTimeStep=1.0, period=0.0, filterInterval=0,
                 boundary=None, closure=False, viscosity=1.0034e-6, shifting=False, shiftingMach=0.1, spacing=None,
                 shiftingLocal=False):
        sp = StepParams()
        sp.dim, sp.kind, sp.period, sp.hMax, sp.hMin = dim, 1 if kernelType == 'wendlandC2' else 0, period, hMax, hMax
        sp.rho0, sp.c0, sp.alpha, sp.boundaryFactor = rho0, c0, alpha, boundaryFactor
        for a, value in enumerate(gravity):
            sp.g[a] = value
        sp.xsphEpsilon, sp.densityFloor = xsphEpsilon, densityFloor
        sp.diffusion, sp.delta = self.diffusionModes[diffusion], delta
        sp.wallExtrapolated, sp.tension, sp.corrected, sp.limited = (int(wallExtrapolated), int(tension),
                                                                    int(corrected), int(limited))
        sp.cfl, sp.maxTimeStep = cfl, maxTimeStep
        sp.closure, sp.viscosity = int(closure), float(viscosity)
        if shifting:
            # src/pysurf/sphSolver.py:258-274: the free surface's thresholds, W(dx) for the anti-clumping
            sp.shifting, sp.shiftLocal, sp.shiftMach = 1, int(shiftingLocal), float(shiftingMach)
            sp.spacingKernel = lib().orx_kernel_value(sp.kind, dim, float(spacing), hMax)
            sp.shiftThreshold = {2: 1.5, 3: 2.4}[dim]
            sp.lopsidedness = 0.4 if kernelType == 'wendlandC2' else 0.3
        self.params, self.filterInterval, self._keep = sp, filterInterval, None
        self.energy = None
        self.setBoundary(boundary)
        self.time, self.step = 0.0, 0

    def trackEnergy(self, enabled=True):
        """Keep the energy budget from now on: `energy` holds each term's total since this call."""
        self.energy = np.zeros(len(ENERGY_TERMS)) if enabled else None
        self.params.energy = self.energy.ctypes.data if enabled else None

    def setBoundary(self, boundary):
        """boundary: None, ('container', lower, upper, openTop), ('bed', BedParams), ('field', FieldParams)."""
        sp = self.params
        sp.boundaryKind = 0
        if boundary is None:
            return
        if boundary[0] == 'container':
            sp.boundaryKind = 1
            for a, (lo, hi) in enumerate(zip(boundary[1], boundary[2])):
                sp.lower[a], sp.upper[a] = lo, hi
            sp.openTop = int(boundary[3])
        elif boundary[0] == 'bed':
            sp.boundaryKind, sp.bed, self._keep = 2, boundary[1], boundary[1]._keep
        elif boundary[0] == 'field':
            sp.boundaryKind, sp.field, self._keep = 3, boundary[1], boundary[1]._keep

    def __call__(self, state):
        """Advance ``state`` (dict with positions, velocities, densities, masses, isFluid, lengths) in place."""
        sp = self.params
        h = state.get('lengths')
        n = len(state['positions'])
        h = np.full(n, sp.hMax) if h is None else _f64(h)
        sp.hMin = float(h.min())
        sp.filterDensity = int(bool(self.filterInterval) and self.step > 0 and self.step % self.filterInterval == 0)
        for key in ('positions', 'velocities', 'densities'):
            state[key] = _f64(state[key])
        state.setdefault('pressures', np.zeros(n))
        state.setdefault('accelerations', np.zeros_like(state['positions']))
        state['pressures'] = _f64(state['pressures'])
        state['accelerations'] = _f64(state['accelerations'])
        dt = lib().or_step(C.byref(sp), n, state['positions'], state['velocities'], state['densities'],
                           _f64(state['masses']), h, _u8a(state['isFluid']), state['pressures'],
                           state['accelerations'])
        self.time += dt
        self.step += 1
        return dt


def splitParticles(state, mask, rho0, referenceLength, lengthRatio=1.0):
    """src/pysurf/sphRefinement.py:136-190 on a dict state: 2^dim daughters, first in place, rest appended."""
    fluid = np.asarray(state['isFluid'], dtype=bool)
    chosen = np.flatnonzero(np.asarray(mask, dtype=bool) & fluid)
    if chosen.size == 0:
        return 0
    x = _f64(state['positions']).copy()
    dim = x.shape[1]
    count = 2 ** dim
    n = len(x)
    lengths = np.full(n, referenceLength) if state.get('lengths') is None else _f64(state['lengths']).copy()
    corners = np.array(list(itertools.product((-0.25, 0.25), repeat=dim)))
    masses = _f64(state['masses']).copy()
    spacing = (masses[chosen] / rho0) ** (1.0 / dim)
    daughters = x[chosen][:, None, :] + spacing[:, None, None] * corners[None]
    mass = masses[chosen] / count
    length = lengths[chosen] * lengthRatio
    x[chosen] = daughters[:, 0]
    masses[chosen] = mass
    lengths[chosen] = length

    def rep(values):
        return np.repeat(values, count - 1, axis=0)

    state['positions'] = np.vstack([x, daughters[:, 1:].reshape(-1, dim)])
    for key in ('velocities', 'accelerations'):
        if key in state:
            state[key] = np.vstack([state[key], rep(_f64(state[key])[chosen])])
    for key in ('densities', 'pressures'):
        if key in state:
            state[key] = np.concatenate([state[key], rep(_f64(state[key])[chosen])])
    state['masses'] = np.concatenate([masses, rep(mass)])
    state['isFluid'] = np.concatenate([fluid, np.ones(chosen.size * (count - 1), dtype=bool)])
    state['lengths'] = np.concatenate([lengths, rep(length)])
    return int(chosen.size)


def crestZone(state, x0, y0, width, nx, ny, threshold, minMass):
    """The crest zone the device splits (sph_split_crest_zone; the zone of BreakingWave3D._refineCrest,
    src/pysurf/BreakingWave3D.py:530-576, read as columns): every fluid particle of mass at least
    minMass whose column -- floor((x - x0) / width), floor((y - y0) / width) in 3D, nx by ny of them --
    has its highest fluid particle above threshold.  Returns the mask."""
    x = _f64(state['positions'])
    dim = x.shape[1]
    fluid = np.asarray(state['isFluid'], dtype=bool)
    cx = np.floor((x[:, 0] - x0) / width)
    cy = np.floor((x[:, 1] - y0) / width) if dim == 3 else np.zeros(len(x))
    inside = fluid & (cx >= 0) & (cx < nx) & (cy >= 0) & (cy < ny)
    column = np.where(inside, cy * nx + cx, 0).astype(np.int64)
    tops = np.full(int(nx * ny), -np.inf)
    np.maximum.at(tops, column[inside], x[inside, dim - 1])
    return inside & (_f64(state['masses']) >= minMass) & (tops[column] > threshold)


def refinementLevels(masses, referenceMass, dim):
    """src/pysurf/sphRefinement.py:123-134: how many times each particle has split, from its mass."""
    return np.rint(np.log2(referenceMass / _f64(masses)) / dim).astype(int)


def _cellGroups(points, cell, offset, size):
    """src/pysurf/sphRefinement.py:192-217: bin the points into cubes `cell` across (the grid moved by
    `offset` cells); in every cube holding `size` or more, the `size` nearest its centre, ties to the
    lower index.  Rows of point indices, the cubes in their raveled order."""
    u = points / cell + offset
    base = np.floor(u)
    keys = base.astype(np.int64)
    keys -= keys.min(axis=0)
    flat = np.ravel_multi_index(keys.T, keys.max(axis=0) + 1)
    off = np.sum((u - base - 0.5) ** 2, axis=1)
    order = np.lexsort((np.arange(len(points)), off, flat))
    cubes, first, counts = np.unique(flat[order], return_index=True, return_counts=True)
    rows = [order[f:f + size] for f, c in zip(first, counts) if c >= size]
    return np.array(rows, dtype=np.int64).reshape(-1, size)


def mergeParticles(state, mask, rho0, referenceMass, referenceLength, lengthRatio=1.0, offsets=(0.0, 0.5)):
    """src/pysurf/sphRefinement.py:219-311 on a dict state: the chosen split fluid particles of each
    level, 2^dim to a cube one level coarser, merge into one at the group's first place; fluid from the
    end fills the places the others leave among the boundary's.  Returns (groups, removed kinetic
    energy, source), source the old index of each particle after."""
    x = _f64(state['positions'])
    n, dim = x.shape
    size = 2 ** dim
    fluid = np.asarray(state['isFluid'], dtype=bool)
    levels = refinementLevels(state['masses'], referenceMass, dim)
    eligible = np.asarray(mask, dtype=bool) & fluid & (levels > 0)
    found = []
    for level in sorted(set(levels[eligible].tolist())):
        cell = (referenceMass / size ** (level - 1) / rho0) ** (1.0 / dim)
        free = np.flatnonzero(eligible & (levels == level))
        for offset in offsets:
            if free.size < size:
                break
            rows = free[_cellGroups(x[free], cell, offset, size)]
            if rows.size:
                found.append(rows)
                free = free[~np.isin(free, rows.ravel())]
    if not found:
        return 0, 0.0, np.arange(n)
    members = np.sort(np.vstack(found), axis=1)
    m = _f64(state['masses'])[members]
    total = m.sum(axis=1)
    w = m / total[:, None]
    v = _f64(state['velocities'])[members]
    mean = np.sum(w[:, :, None] * v, axis=1)
    removed = 0.5 * float(np.sum(m * np.sum((v - mean[:, None, :]) ** 2, axis=2)))
    lengths = np.full(n, referenceLength) if state.get('lengths') is None else _f64(state['lengths']).copy()
    head = members[:, 0]
    out = {key: np.array(state[key], dtype=float) for key in ('positions', 'velocities', 'accelerations',
                                                               'densities', 'pressures', 'masses')}
    out['positions'][head] = np.sum(w[:, :, None] * x[members], axis=1)
    out['accelerations'][head] = np.sum(w[:, :, None] * _f64(state['accelerations'])[members], axis=1)
    out['pressures'][head] = np.sum(w * _f64(state['pressures'])[members], axis=1)
    out['densities'][head] = total / np.sum(m / _f64(state['densities'])[members], axis=1)
    out['velocities'][head] = mean
    out['masses'][head] = total
    lengths[head] = lengths[members].mean(axis=1) / lengthRatio
    out['lengths'] = lengths
    out['isFluid'] = fluid.copy()
    # the compaction: the group's others go; fluid from the end takes the places among the boundary's
    gone = np.zeros(n, dtype=bool)
    gone[members[:, 1:].ravel()] = True
    last = int(np.flatnonzero(~fluid).max()) if (~fluid).any() else -1
    holes = np.flatnonzero(gone[:last + 1])
    tail = np.flatnonzero(~gone[last + 1:]) + last + 1
    if tail.size < holes.size:
        raise RuntimeError('too few fluid particles after the boundary to fill its places')
    movers = tail[tail.size - holes.size:]
    keep = ~gone
    keep[holes] = True
    keep[movers] = False
    source = np.arange(n)
    source[holes] = movers
    source = source[keep]
    for key, values in out.items():
        state[key] = values[source]
    return int(len(members)), removed, source
