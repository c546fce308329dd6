"""The energy budget's restatement in the oracle against the reference's own budget.

src/pysurf/sphEnergy.py defines the elastic energy, its secant slope and the terms; the reference's
array solver keeps them step by step (src/pysurf/sphSolver.py:1650-1852, 1909-1936) and its device
steps per particle (src/pysurf/sphGpu.py:303-545, 1046-1230).  The fixtures (tests/golden/energy.npz)
are the array solver's budgets over the reference's own energy runs (tests/testSphEnergy.py) and over
sloshing runs that reach the Shepard filter, wall viscosity, shifting, the clamp and the floor.
"""
import numpy as np
import pytest
from scipy.integrate import quad

from conftest import golden
from oracle import oracle
from test_oracle_golden import stepperFor

ENERGY = np.load('tests/golden/energy.npz')
RUNS = ['channel', 'uncorrected', 'published', 'hybrid', 'filtered', 'shifted', 'clamped']
NU = 1.0034e-6      # the closure's water viscosity, as the runs' configuration carries it


def test_terms_are_the_references():
    assert tuple(ENERGY['terms'][:14]) == oracle.ENERGY_TERMS
    assert ENERGY['terms'][14] == 'refinement'


@pytest.mark.parametrize('tension', [False, True])
def test_elastic_energy_and_slope_match_the_reference(tension):
    rho0, c0 = float(ENERGY['elastic/rho0']), float(ENERGY['elastic/c0'])
    e = oracle.elasticEnergy(ENERGY['elastic/densities'], rho0, c0, tension)
    assert np.allclose(e, ENERGY[f'elastic/energy_{int(tension)}'], rtol=1e-13, atol=1e-300)
    slope = oracle.elasticSlope(ENERGY['elastic/before'], ENERGY['elastic/after'], rho0, c0, tension)
    assert np.allclose(slope, ENERGY[f'elastic/slope_{int(tension)}'], rtol=1e-9, atol=1e-300)


@pytest.mark.parametrize('tension', [False, True])
def test_elastic_energy_is_the_integral_of_pressure_over_density_squared(tension):
    # tests/testSphEnergy.py:72-80
    rho0, c0 = 1000.0, 20.0

    def pressure(s):
        p = rho0 * c0 ** 2 / 7.0 * ((s / rho0) ** 7 - 1.0)
        return p if tension else max(p, 0.0)

    for density in (985.0, 999.0, 1000.0, 1000.2, 1003.0, 1030.0):
        integral, _ = quad(lambda s: pressure(s) / s ** 2, rho0, density, epsabs=1e-14, epsrel=1e-12)
        assert float(oracle.elasticEnergy(density, rho0, c0, tension)[0]) == pytest.approx(integral, rel=1e-9,
                                                                                          abs=1e-15)


def budgetRun(tag):
    """The oracle's steps over a fixture run with the budget on: (budget, start energy, end energy, state)."""
    r = golden('energy.npz', tag)
    mach, spacing = float(r['shifting'][1]), float(r['shifting'][2])
    stepper = stepperFor(r, closure=bool(r['closure']), viscosity=NU, shifting=bool(r['shifting'][0]),
                         shiftingMach=mach, spacing=spacing)
    sp = stepper.params
    state = {k: r[k].copy() for k in ('positions', 'velocities', 'densities', 'masses', 'isFluid')}
    energy = lambda: oracle.fluidEnergy(state, r['gravity'], sp.rho0, sp.c0, bool(sp.tension))   # noqa: E731
    start = energy()
    stepper.trackEnergy()
    dts = [stepper(state) for _ in range(int(r['steps']))]
    assert np.allclose(dts, r['dts'], rtol=1e-10, atol=0.0)
    return r, stepper.energy.copy(), start, energy(), state


@pytest.mark.parametrize('tag', RUNS)
def test_the_budget_matches_the_references_and_closes(tag):
    r, budget, start, end, state = budgetRun(tag)
    expected = r['budget'][:14]
    scale = np.abs(r['budget']).sum()
    # the fluid's energies are the reference's at the start and at the end
    assert np.allclose(start, r['startEnergy'], rtol=1e-12, atol=1e-12 * scale)
    assert np.allclose(end, r['endEnergy'], rtol=1e-9, atol=1e-9 * scale)
    # each term is the reference's: the device form and the array form differ only in rounding
    for k, name in enumerate(oracle.ENERGY_TERMS):
        assert budget[k] == pytest.approx(expected[k], abs=1e-9 * scale), name
    # and the terms close on the change of K + P + E_C (tests/testSphEnergy.py:93-110)
    assert budget.sum() == pytest.approx((end - start).sum(), abs=1e-9 * np.abs(budget).sum())


def test_a_planted_mistake_breaks_the_closure():
    # the budget's check on itself: drop the floor's term and a run that floors no longer closes
    r, budget, start, end, state = budgetRun('clamped')
    k = oracle.ENERGY_TERMS.index('floor')
    assert abs(budget[k]) > 1e-3 * np.abs(budget).sum()
    assert abs(budget.sum() - budget[k] - (end - start).sum()) > 1e-6 * np.abs(budget).sum()
