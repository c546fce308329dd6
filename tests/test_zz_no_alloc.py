"""The allocation-free entry point against the library's own path, on the GPU.

``sph_fluid_maxima_noalloc`` serves callers that cannot let the library allocate device memory
(an application whose memory is all held by its own pool allocator, or a loop that must not
enter the CUDA allocator while it runs): it reads the caller's device arrays and keeps its
scratch in a fixed file-scope device array.  Its maxima must equal those the momentum sweep
reduces (``PairSums.residentRates``) and its time step the reference's cflTimeStep, on two calls
in a row (the second finds the first call's scratch and must clear what it needs).

This file sorts last so that a run stopping at the first failure has run every other test.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_no_alloc_maxima_match_the_momentum_sweeps():
    import torch

    from pysurf_b200 import _lib, cases

    case = cases.solitaryBeach(particlesPerDepth=16)
    sums = cases.pairSumsFor(case)
    state = case.state.copy()
    sums.push(state)
    sums.setBoundary(case.boundary, state)
    sums.advance(0.0, 0, math.inf, 3, case.smoothingLength, case.cflNumber, case.maxTimeStep)
    vmax, amax = sums.residentRates(False)          # the sweep's own reduction, at the current state
    out = sums.pullState()
    h, c0, cfl, maxdt = case.smoothingLength, case.soundSpeed, case.cflNumber, case.maxTimeStep
    dt = cfl * h / (c0 + vmax)
    if amax > 1e-12:
        dt = min(dt, cfl * math.sqrt(h / amax))
    dt = min(dt, maxdt)

    # the caller's own device arrays: allocated by the caller (torch here), not by the entry point
    device = torch.device('cuda', 0)
    velocities = torch.tensor(out['velocities'], dtype=torch.float64, device=device).contiguous()
    accelerations = torch.tensor(out['accelerations'], dtype=torch.float64, device=device).contiguous()
    fluid = torch.tensor(out['isFluid'].astype(np.uint8), dtype=torch.uint8, device=device).contiguous()
    result = torch.zeros(3, dtype=torch.float64, device=device)
    lib = _lib.load()
    stream = torch.cuda.current_stream(device).cuda_stream
    n = len(out['masses'])
    for call in range(2):
        result.fill_(-1.0)
        status = lib.sph_fluid_maxima_noalloc(velocities.data_ptr(), accelerations.data_ptr(), fluid.data_ptr(), n,
                                              2, h, c0, cfl, maxdt, result.data_ptr(), stream)
        assert status == 0, lib.sph_last_error().decode()
        torch.cuda.synchronize(device)
        got = result.cpu().numpy()
        assert got[0] == pytest.approx(vmax, rel=1e-15, abs=0.0), call
        assert got[1] == pytest.approx(amax, rel=1e-15, abs=0.0), call
        assert got[2] == pytest.approx(dt, rel=1e-15, abs=0.0), call

    # sizes past the fixed scratch are refused before anything is launched
    status = lib.sph_fluid_maxima_noalloc(velocities.data_ptr(), accelerations.data_ptr(), fluid.data_ptr(),
                                          16_777_217, 2, h, c0, cfl, maxdt, result.data_ptr(), stream)
    assert status == _lib.SPH_ERR_INVALID
    assert 'exceed' in lib.sph_last_error().decode()
