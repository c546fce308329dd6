"""The C-ABI over device arrays: a state pushed from torch CUDA tensors and pulled back into them
(sph_push_device, sph_pull_device) steps exactly as one pushed from host arrays; a pull right after
a push gives the state's Tait pressures; the loaded kernels are sm_100a code."""
import ctypes
import math

import numpy as np
import pytest

from pysurf_b200 import _lib, cases

pytestmark = pytest.mark.gpu


def test_the_loaded_kernels_are_sm_100a():
    version = ctypes.c_int(0)
    _lib.check(_lib.load().sph_kernel_architecture(ctypes.byref(version)), 'sph_kernel_architecture')
    assert version.value == 100


def _run(case, push, pull, steps=20):
    sums = cases.pairSumsFor(case)
    push(sums)
    sums.setBoundary(case.boundary, case.state)
    t, step, _ = sums.advance(0.0, 0, math.inf, steps, case.smoothingLength, case.cflNumber, case.maxTimeStep,
                              case.densityFilterInterval)
    assert step == steps
    return t, pull(sums)


def test_a_state_pushed_and_pulled_through_device_tensors_steps_as_the_host_one():
    import torch
    case = cases.solitaryBeach(particlesPerDepth=8)
    st = case.state
    fields = ('positions', 'velocities', 'densities', 'pressures', 'accelerations')

    def hostPush(sums):
        sums.push(st.copy())

    def hostPull(sums):
        out = st.copy()
        sums.pull(out)
        return {k: np.array(getattr(out, k)) for k in fields}

    dev = torch.device('cuda:0')
    tensors = {k: torch.tensor(np.asarray(getattr(st, k), dtype=np.float64), device=dev)
               for k in ('positions', 'velocities', 'densities')}
    masses = torch.tensor(np.broadcast_to(st.masses, (st.nParticles,)).astype(np.float64), device=dev)
    flags = torch.tensor(np.asarray(st.isFluid, dtype=np.uint8), device=dev)

    def devicePush(sums):
        sums.pushDevice(tensors['positions'], tensors['velocities'], tensors['densities'], masses, flags)

    def devicePull(sums):
        n, dim = st.nParticles, case.dimensions
        out = {k: torch.full((n, dim) if k in ('positions', 'velocities', 'accelerations') else (n,), math.nan,
                             dtype=torch.float64, device=dev) for k in fields}
        extra = {'masses': torch.zeros(n, dtype=torch.float64, device=dev),
                 'isFluid': torch.zeros(n, dtype=torch.uint8, device=dev)}
        sums.pullDevice(**out, **extra)
        assert np.array_equal(extra['masses'].cpu().numpy(), np.broadcast_to(st.masses, (n,)))
        assert np.array_equal(extra['isFluid'].cpu().numpy().astype(bool), np.asarray(st.isFluid, dtype=bool))
        return {k: v.cpu().numpy() for k, v in out.items()}

    t0, a = _run(case, hostPush, hostPull)
    t1, b = _run(case, devicePush, devicePull)
    assert t0 == t1
    for k in fields:
        assert np.array_equal(a[k], b[k]), k


def test_device_tensors_are_checked_before_any_copy():
    import torch
    case = cases.solitaryBeach(particlesPerDepth=8)
    st = case.state
    n = st.nParticles
    sums = cases.pairSumsFor(case)
    x = torch.tensor(st.positions, device='cuda:0')
    v = torch.tensor(st.velocities, device='cuda:0')
    rho = torch.tensor(st.densities, device='cuda:0')
    m = torch.full((n,), float(np.mean(st.masses)), dtype=torch.float64, device='cuda:0')
    fl = torch.tensor(np.asarray(st.isFluid, dtype=np.uint8), device='cuda:0')
    with pytest.raises(ValueError):
        sums.pushDevice(x.float(), v, rho, m, fl)            # float32 positions
    with pytest.raises(ValueError):
        sums.pushDevice(x.cpu(), v, rho, m, fl)              # host tensor
    with pytest.raises(ValueError):
        sums.pushDevice(x[:, :1], v, rho, m, fl)             # wrong shape
    with pytest.raises(ValueError):
        sums.pushDevice(x, v, rho, m, fl, torch.full((n,), 2.0 * case.smoothingLength, dtype=torch.float64,
                                                      device='cuda:0'))   # a length beyond the grid's h


def test_a_pull_right_after_a_push_gives_tait_pressures_and_no_accelerations():
    case = cases.solitaryBeach(particlesPerDepth=8)
    st = case.state.copy()
    sums = cases.pairSumsFor(case)
    sums.push(st)
    out = case.state.copy()
    out.pressures = np.full(st.nParticles, np.nan)
    out.accelerations = np.full((st.nParticles, case.dimensions), np.nan)
    sums.pull(out)
    rho0, c0 = case.referenceDensity, case.soundSpeed
    tait = np.maximum(rho0 * c0 * c0 / 7.0 * ((st.densities / rho0) ** 7 - 1.0), 0.0)
    assert np.allclose(out.pressures, tait.astype(np.float32), rtol=1e-6, atol=1e-3)
    assert np.array_equal(out.accelerations, np.zeros_like(out.accelerations))
    np.testing.assert_array_equal(out.densities, st.densities)
