"""A push of more than a million lengths, which the library scans on several host threads: a length
past the grid's h or not positive is refused wherever it lies, and so are mixed lengths while
shifting is on (src/pysurf/sphGpu.py:1998-2042 raises for both).  The C-ABI is called directly, so
the Python wrapper's own range check does not decide first."""
import numpy as np
import pytest

from pysurf_b200 import _lib
from pysurf_b200.sphGpu import PairSums

pytestmark = pytest.mark.gpu

N = 1_200_000       # above the size from which the scan takes several threads
H = 0.03


def _cloud():
    rng = np.random.default_rng(3)
    return (rng.uniform(0.0, 1.0, (N, 3)), np.zeros((N, 3)), np.full(N, 1000.0), np.full(N, 1e-3),
            np.ones(N, dtype=np.uint8))


def _push(sums, cloud, lengths):
    positions, velocities, densities, masses, fluid = cloud
    return sums._lib.sph_push(sums._handle, N, _lib.dptr(positions), _lib.dptr(velocities), _lib.dptr(densities),
                              _lib.dptr(masses), fluid.ctypes.data_as(_lib._pu8), _lib.dptr(lengths))


@pytest.mark.parametrize('where', [0, N // 2, N - 1])
def test_a_length_past_h_or_not_positive_is_refused_wherever_it_lies(where):
    sums = PairSums(3, H, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    cloud = _cloud()
    lengths = np.full(N, H)
    assert _push(sums, cloud, lengths) == _lib.SPH_OK
    lengths[where] = 1.5 * H
    assert _push(sums, cloud, lengths) == _lib.SPH_ERR_INVALID
    lengths[where] = -H
    assert _push(sums, cloud, lengths) == _lib.SPH_ERR_INVALID
    lengths[where] = 0.5 * H
    assert _push(sums, cloud, lengths) == _lib.SPH_OK


@pytest.mark.parametrize('where', [0, N // 3, N - 1])
def test_one_shorter_length_anywhere_is_refused_while_shifting(where):
    sums = PairSums(3, H, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    sums.setShifting(True, 0.1, H / 3.0, 20.0)
    cloud = _cloud()
    lengths = np.full(N, H)
    assert _push(sums, cloud, lengths) == _lib.SPH_OK
    lengths[where] = 0.5 * H
    assert _push(sums, cloud, lengths) == _lib.SPH_ERR_INVALID
