"""ctypes binding of libpysurf_b200.so, the C-ABI declared in include/pysurf_b200.h.

The library is loaded from this package's directory, where ``pysurf_b200.build`` puts it.
There is no fallback: if the library is missing or a call fails, an exception says so.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(HERE, 'libpysurf_b200.so')

SPH_OK = 0
SPH_ERR_INVALID = -1
SPH_ERR_NOMEM = -2
SPH_ERR_CUDA = -3
SPH_ERR_NONFINITE = -4
SPH_ERR_TIMESTEP = -5
SPH_ERR_STATE = -6
SPH_ERR_CAPACITY = -7
SPH_ERR_UNSUPPORTED = -8

# Every entry point of include/pysurf_b200.h with its argument types; the tests check the
# library exports each of these names.
_d, _i, _i64, _vp = C.c_double, C.c_int, C.c_int64, C.c_void_p
_pd = C.POINTER(C.c_double)
_pi64 = C.POINTER(C.c_int64)
_pu8 = C.POINTER(C.c_uint8)
_pi32 = C.POINTER(C.c_int32)
_pf = C.POINTER(C.c_float)
_h = C.c_void_p

SIGNATURES = {
    'sph_create': [_i, _d, _pd, _pd, _d, _i, _i, _i, C.POINTER(C.c_void_p)],
    'sph_destroy': [_h],
    'sph_last_error': [],
    'sph_version': [],
    'sph_kernel_architecture': [C.POINTER(C.c_int)],
    'sph_grid_shape': [_h, _pi64],
    'sph_set_cells_per_support': [_h, _i],
    'sph_set_stream': [_h, _vp],
    'sph_set_sweep_options': [_h, _i, _i],
    'sph_neighbor_table': [_h, _pi64],
    'sph_set_diffusion': [_h, _i, _d, _d, _d, _d],
    'sph_set_wall_pressure': [_h, _i],
    'sph_set_negative_pressure': [_h, _i],
    'sph_set_continuity_correction': [_h, _i],
    'sph_set_viscosity_limiter': [_h, _i],
    'sph_set_physics': [_h, _d, _d, _d, _d, _pd, _d, _d],
    'sph_update': [_h, _i64, _pd, _pd, _pu8, _pd],
    'sph_pair_accelerations': [_h, _pd, _pd, _pd, _d, _d, _d, _pd, _pd],
    'sph_continuity_rate': [_h, _pd, _pd, _pd],
    'sph_xsph_velocity': [_h, _pd, _pd, _d, _pd],
    'sph_wall_pressure': [_h, _pd, _pd, _pd, _d, _d, _pd],
    'sph_shepard_density': [_h, _pd, _pd],
    'sph_velocity_gradients': [_h, _pd, _pd, _pd],
    'sph_correction_matrices': [_h, _pd, _pd],
    'sph_density_gradients': [_h, _pd, _pd],
    'sph_push': [_h, _i64, _pd, _pd, _pd, _pd, _pu8, _pd],
    'sph_pull': [_h, _pd, _pd, _pd, _pd, _pd, _pd, _pd, _pu8],
    'sph_push_device': [_h, _i64, _vp, _vp, _vp, _vp, _vp, _vp],
    'sph_pull_device': [_h, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    'sph_count': [_h, _pi64],
    'sph_frame': [_h, _pf, _pf, _pu8],
    'sph_clear_boundary': [_h],
    'sph_set_boundary_container': [_h, _pd, _pd, _i],
    'sph_set_boundary_bed': [_h, _pd, _pd, _i64, _d, _i, _d, _i, _d, _d, _d],
    'sph_set_boundary_height_field': [_h, _pd, _i64, _i64, _d, _d, _d, _d, _d, _d, _d, _i, _d, _d],
    'sph_enforce_boundary': [_h],
    'sph_resident_rates': [_h, _i, _pd, _pd],
    'sph_resident_integrate': [_h, _d],
    'sph_advance': [_h, _pd, _pi64, _pd, _d, _i64, _d, _d, _d, _i64],
    'sph_cell_order_key': [_pd, _i64, _i, _d, _pi64, _pi64, _i],
    'sph_neighbor_list': [_h, _d, _pi64, _pi32, _i64, _pi64],
    'sph_split': [_h, _pu8, _d, _d, _pi64],
    'sph_merge': [_h, _pu8, _d, _d, _d, _pi64, _pd, _pi64],
    'sph_set_closure': [_h, _i, _d, _d, _d],
    'sph_set_shifting': [_h, _i, _d, _d, _d, _i],
    'sph_shifting_displacement': [_h, _pd, _d, _pd, _pd, _pd, _pd],
    'sph_set_energy_budget': [_h, _i],
    'sph_set_compensated_sums': [_h, _i],
    'sph_energy_sums': [_h, _pd],
    'sph_fluid_energy': [_h, _pd],
    'sph_closure_coefficients': [_h, _pd, _pd, _pd, _pd],
    'sph_surface_tops': [_h, _d, _d, _i64, _pd],
    'sph_split_crest_zone': [_h, _d, _d, _d, _i64, _i64, _d, _d, _d, _d, _pi64],
    'sph_face_cells': [_h, _d, _d, _d, _d, _d, _d, _d, _i64, _i64, _pu8],
    'sph_bed_sheet': [_h, _pd, _pd, _i64, _d, _pd, _i64, _pi64],
    'sph_section_tops': [_h, _d, _d, _d, _d, _i64, _pd],
    'sph_section_face_cells': [_h, _d, _d, _d, _d, _d, _d, _d, _d, _d, _i64, _i64, _pu8],
    'sph_section_bed_sheet': [_h, _d, _d, _pd, _pd, _i64, _d, _pd, _i64, _pi64],
    'sph_last_advance_ms': [_h, _pd],
    'sph_begin_steps': [_h, _d, _i64, _d, _d, _i64, _d, _d, _d, _i64],
    'sph_enqueue_steps': [_h, _i64],
    'sph_finish_steps': [_h, _pd, _pi64, _pd],
    'sph_stage_times': [_h, _pd, _i64, _pi64],
    'sph_stage_name': [_i64],
    'sph_step_launches': [_h, _pi64],
    'sph_fluid_maxima_noalloc': [_vp, _vp, _vp, _i64, _i, _d, _d, _d, _d, _vp, _vp],
}


class SphError(RuntimeError):
    """A failure reported by the CUDA backend, with its status code."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


_lib = None


def load():
    """The loaded library; raises ImportError when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBRARY):
        raise ImportError(f'{LIBRARY} is missing: build it with `python -m pysurf_b200.build` (nvcc, sm_100a).')
    lib = C.CDLL(LIBRARY)
    for name, argtypes in SIGNATURES.items():
        function = getattr(lib, name)
        function.argtypes = argtypes
        function.restype = C.c_char_p if name in ('sph_last_error', 'sph_stage_name') else C.c_int
    _lib = lib
    return lib


def check(status: int, what: str = '') -> None:
    """Raise the backend's error for a failed call: ValueError for bad arguments, SphError otherwise."""
    if status == SPH_OK:
        return
    message = load().sph_last_error().decode(errors='replace')
    text = f'{what}: {message}' if what else message
    if status == SPH_ERR_INVALID:
        raise ValueError(text)
    raise SphError(status, text)


def dptr(array):
    """A float64 pointer into a C-contiguous numpy array, or None."""
    if array is None:
        return None
    assert array.dtype == np.float64 and array.flags['C_CONTIGUOUS']
    return array.ctypes.data_as(_pd)


def f64(array, shape=None):
    """A C-contiguous float64 copy (or view) of an array, checked against a shape."""
    out = np.ascontiguousarray(array, dtype=np.float64)
    if shape is not None and out.shape != tuple(shape):
        raise ValueError(f'expected shape {tuple(shape)}, got {out.shape}')
    return out


def u8(array):
    """A C-contiguous uint8 view of a flag array (a bool array's own memory, so pinned stays pinned)."""
    out = np.ascontiguousarray(np.asarray(array).astype(bool, copy=False).view(np.uint8))
    return out, out.ctypes.data_as(_pu8)
