"""The oracle's restatement of mergeParticles (src/pysurf/sphRefinement.py:192-311) against merges the
reference made (tests/golden/merge.npz): lattices with their boundary, split in part with h kept or
halved, once or twice, jittered, and merged in part."""
import numpy as np
import pytest

from oracle import oracle

MERGE = np.load('tests/golden/merge.npz')
TAGS = sorted({k.split('/')[0] for k in MERGE.files})
FIELDS = ('positions', 'velocities', 'accelerations', 'densities', 'pressures', 'masses', 'isFluid', 'lengths')


@pytest.mark.parametrize('tag', TAGS)
def test_the_oracle_merges_as_the_reference(tag):
    state = {name: MERGE[f'{tag}/{name}'].copy() for name in FIELDS}
    rho0, referenceMass, length, ratio = MERGE[f'{tag}/reference']
    groups, removed, source = oracle.mergeParticles(state, MERGE[f'{tag}/mask'], rho0, referenceMass, length, ratio)
    assert groups == int(MERGE[f'{tag}/groups'])
    assert np.array_equal(source, MERGE[f'{tag}/source'])
    assert removed == pytest.approx(float(MERGE[f'{tag}/removedEnergy']), rel=1e-12)
    for name in ('masses', 'isFluid', 'lengths'):
        assert np.array_equal(state[name], MERGE[f'{tag}/merged_{name}']), name
    for name in ('positions', 'velocities', 'accelerations', 'densities', 'pressures'):
        assert np.allclose(state[name], MERGE[f'{tag}/merged_{name}'], rtol=1e-14, atol=1e-14), name


def test_the_boundary_keeps_its_places():
    # the reference's own rule (src/pysurf/sphRefinement.py:288-303): every boundary index holds
    for tag in TAGS:
        boundary = np.flatnonzero(~MERGE[f'{tag}/isFluid'])
        assert not MERGE[f'{tag}/merged_isFluid'][boundary].any()
        assert np.array_equal(MERGE[f'{tag}/merged_positions'][boundary], MERGE[f'{tag}/positions'][boundary])
