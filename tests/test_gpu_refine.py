"""Crest-zone refinement on the device (sph_split_crest_zone): the zone against the same columns
taken on the host from pulled positions, the split exact in mass, and mixed-h steps after it."""
import math

import numpy as np
import pytest

from pysurf_b200 import cases

pytestmark = pytest.mark.gpu


def hostZone(state, case, share=0.3):
    info, s = case.info, case.spacing
    depth, height = float(info['depth']), float(info['H/d']) * float(info['depth'])
    lower, upper = case.domainMin, case.domainMax
    dim = case.dimensions
    nx = int(math.ceil((upper[0] - lower[0]) / s))
    ny = int(math.ceil((upper[1] - lower[1]) / s)) if dim == 3 else 1
    x = state['positions']
    fluid = state['isFluid']
    cx = np.floor((x[:, 0] - lower[0]) / s)
    cy = np.floor((x[:, 1] - lower[1]) / s) if dim == 3 else np.zeros(len(x))
    inside = fluid & (cx >= 0) & (cx < nx) & (cy >= 0) & (cy < ny)
    column = (cy * nx + cx).astype(np.int64)
    tops = np.full(nx * ny, -np.inf)
    np.maximum.at(tops, column[inside], x[inside, dim - 1])
    fluidMass = float(np.max(case.state.masses[case.state.isFluid]))
    return inside & (state['masses'] >= 0.999 * fluidMass) & (tops[np.where(inside, column, 0)] > depth + share * height)


@pytest.mark.parametrize('build', [lambda: cases.solitaryBeach(16), lambda: cases.ridgeWave3D(6)])
def test_the_device_crest_zone_splits_what_the_host_zone_selects(build):
    case = build()
    sums = cases.pairSumsFor(case)
    state = case.state.copy()
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    t, step, dt = sums.advance(0.0, 0, math.inf, 10, case.smoothingLength, case.cflNumber, case.maxTimeStep)
    before = sums.pullState()
    zone = hostZone(before, case)
    assert zone.any()
    split = cases.refineCrestZone(sums, case)
    assert split == int(zone.sum())
    after = sums.pullState()
    n, dim = len(zone), case.dimensions
    assert len(after['masses']) == n + split * (2 ** dim - 1)
    assert after['masses'].sum() == pytest.approx(before['masses'].sum(), rel=1e-15)
    assert np.array_equal(after['masses'][:n][zone], before['masses'][zone] / 2 ** dim)
    assert np.array_equal(after['masses'][:n][~zone], before['masses'][~zone])
    assert np.all(after['lengths'][:n][zone] == 0.5 * case.smoothingLength)
    assert np.all(after['isFluid'][n:])
    # a second pass finds the zone already split
    assert cases.refineCrestZone(sums, case) == 0
    # mixed-h steps run
    t, step, dt = sums.advance(t, step, math.inf, step + 10, 0.5 * case.smoothingLength, case.cflNumber,
                               case.maxTimeStep, 0, dt)
    final = sums.pullState()
    assert np.all(np.isfinite(final['positions'])) and step == 20


def test_a_split_straight_after_a_push_sizes_the_table_from_a_fresh_cell_list():
    # the daughters have no cell until the next sort: sizing the table must not read the old list
    case = cases.ridgeWave3D(6)
    sums = cases.pairSumsFor(case)
    state = case.state.copy()
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    capacity = sums.neighborTableCapacity()
    assert cases.refineCrestZone(sums, case) > 0
    t, step, dt = sums.advance(0.0, 0, math.inf, 3, 0.5 * case.smoothingLength, case.cflNumber, case.maxTimeStep)
    assert step == 3
    # mother-sized particles beside the split zone meet eight times the daughters: rows grow
    assert sums.neighborTableCapacity() > capacity
