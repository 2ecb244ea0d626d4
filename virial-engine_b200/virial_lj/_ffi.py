"""ctypes declarations of include/virial_lj.h (the library's C ABI)."""

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvirial_lj.so")

PARTICLE = np.dtype([("pos", "<f8", (3,)), ("vel", "<f8", (3,))], align=True)
assert PARTICLE.itemsize == 48


class Thermostat(C.Structure):
    _fields_ = [("kind", C.c_int32), ("temperature", C.c_double), ("friction", C.c_double),
                ("seed", C.c_uint32), ("period", C.c_double)]


class Settings(C.Structure):
    _fields_ = [("box_size", C.c_double * 3), ("cutoff", C.c_double), ("dt", C.c_double),
                ("thermostat", Thermostat), ("shifted_force", C.c_int32), ("skin", C.c_double),
                ("profile_bins", C.c_uint32)]


class Measurement(C.Structure):
    _fields_ = [("step", C.c_uint64), ("time", C.c_double), ("kinetic", C.c_double),
                ("potential", C.c_double), ("virial", C.c_double), ("momentum", C.c_double * 3),
                ("count", C.c_uint32), ("volume", C.c_double), ("list_rebuilds", C.c_uint32),
                ("list_overflow", C.c_uint32), ("thermostat_energy", C.c_double),
                ("condensed", C.c_uint32), ("list_capacity", C.c_uint32),
                ("list_grows", C.c_uint32)]


class Slab(C.Structure):
    _fields_ = [("z", C.c_double), ("particles", C.c_double), ("kinetic", C.c_double * 3),
                ("virial", C.c_double * 3), ("potential", C.c_double)]


class HeatExchange(C.Structure):
    _fields_ = [("hot", C.c_double * 2), ("cold", C.c_double * 2), ("energy", C.c_double)]


class ReplicaDesc(C.Structure):
    _fields_ = [("particles", C.c_void_p), ("count", C.c_size_t), ("box_size", C.c_double * 3),
                ("thermostat", Thermostat)]


class GridInfo(C.Structure):
    _fields_ = [("cells", C.c_uint32 * 3), ("total_cells", C.c_uint32), ("capacity", C.c_uint32),
                ("segment", C.c_uint32), ("rebuilds", C.c_uint32), ("reorder_every", C.c_uint32),
                ("cell_size", C.c_float * 3), ("list_r2", C.c_float)]


STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "BOX_TOO_SMALL", 3: "LIST_OVERFLOW", 4: "CUDA_ERROR",
                5: "TIMEOUT", 6: "BUSY", 7: "NOT_ENABLED", 8: "FULL", 9: "NO_DEVICE"}

_vp = C.c_void_p
_st = C.c_int
_P = C.POINTER

# name -> argument types; every function returns vlj_status (int)
SIGNATURES = {
    "vlj_device_count": [_P(C.c_int)],
    "vlj_create": [_vp, C.c_size_t, _P(Settings), _vp, _P(_vp)],
    "vlj_destroy": [_vp],
    "vlj_step": [_vp, C.c_uint32],
    "vlj_run": [_vp, C.c_uint64],
    "vlj_measure": [_vp, _P(C.c_int)],
    "vlj_poll": [_vp, _P(Measurement), C.c_size_t, _P(C.c_size_t)],
    "vlj_measure_now": [_vp, _P(Measurement)],
    "vlj_read_particles": [_vp, _vp],
    "vlj_write_particles": [_vp, _vp, C.c_size_t],
    "vlj_count": [_vp, _P(C.c_uint32)],
    "vlj_box_size": [_vp, _P(C.c_double)],
    "vlj_volume": [_vp, _P(C.c_double)],
    "vlj_steps": [_vp, _P(C.c_uint64)],
    "vlj_time": [_vp, _P(C.c_double)],
    "vlj_target_temperature": [_vp, _P(C.c_int), _P(C.c_double)],
    "vlj_positions": [_vp, _P(_vp), _P(C.c_size_t)],
    "vlj_velocities": [_vp, _P(_vp)],
    "vlj_set_drawn": [_vp, C.c_int],
    "vlj_set_condensed_neighbours": [_vp, C.c_uint32],
    "vlj_set_temperature": [_vp, C.c_double],
    "vlj_set_heat_exchange": [_vp, _P(HeatExchange)],
    "vlj_heat_flux": [_vp, _P(C.c_int), _P(C.c_double)],
    "vlj_set_grid_every_step": [_vp, C.c_int],
    "vlj_set_list_growth": [_vp, C.c_int],
    "vlj_set_tile_cols": [_vp, C.c_uint32],
    "vlj_sample_profile": [_vp],
    "vlj_clear_profile": [_vp],
    "vlj_read_profile": [_vp, _P(Slab), _P(C.c_double), _P(C.c_uint64)],
    "vlj_record_heat_current": [_vp, C.c_uint32],
    "vlj_sample_heat_current": [_vp],
    "vlj_read_heat_current": [_vp, _P(C.c_double), C.c_size_t, _P(C.c_size_t)],
    "vlj_lattice": [C.c_size_t, C.c_double, C.c_double, C.c_uint64, _vp],
    "vlj_lattice_box": [C.c_size_t, _P(C.c_double), C.c_double, C.c_uint64, _vp],
    "vlj_lattice_fcc": [C.c_uint32, C.c_double, C.c_double, C.c_uint64, _vp, _P(C.c_double)],
    "vlj_profile_interfaces": [_P(C.c_double), C.c_size_t, C.c_double, C.c_double, _P(C.c_double),
                               C.c_size_t, _P(C.c_size_t)],
    "vlj_profile_phases": [_P(C.c_double), C.c_size_t, C.c_double, C.c_double, C.c_double,
                           _P(C.c_int32)],
    "vlj_batch_create": [_P(ReplicaDesc), C.c_size_t, C.c_double, C.c_double, C.c_double, C.c_int32,
                         _vp, _P(_vp)],
    "vlj_batch_destroy": [_vp],
    "vlj_batch_step": [_vp, C.c_uint32],
    "vlj_batch_measure": [_vp, _P(Measurement)],
    "vlj_batch_read_particles": [_vp, C.c_size_t, _vp],
    "vlj_batch_count": [_vp, _P(C.c_size_t), _P(C.c_uint64)],
    "vlj_batch_run": [_vp, C.c_uint64],
    "vlj_batch_box_size": [_vp, C.c_size_t, _P(C.c_double)],
    "vlj_debug_batch_sim": [_vp, _P(_vp)],
    "vlj_debug_grid_info": [_vp, _P(GridInfo)],
    "vlj_debug_read_grid": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "vlj_debug_force_rebuild": [_vp],
    "vlj_debug_read_partials": [_vp, _vp, _vp, _vp],
    "vlj_debug_launches": [_P(C.c_uint64)],
    "vlj_debug_kernels_executed": [_vp, _P(C.c_uint64)],
    "vlj_debug_set_graphs": [_vp, C.c_int],
    "vlj_debug_read_vel4": [_vp, _vp],
    "vlj_debug_kernel_timing": [_vp, C.c_int],
    "vlj_debug_kernel_time": [_vp, _P(C.c_double), _P(C.c_uint64)],
    "vlj_debug_fp32_peak": [_P(C.c_double)],
    "vlj_debug_philox": [_vp, _vp, C.c_size_t, _vp, _vp],
    "vlj_grain_cells": [C.c_double, C.c_double, _P(C.c_uint32)],
    "vlj_grain_contacts": [_vp, _vp, C.c_size_t, C.c_double, C.c_uint32, C.c_uint32, _vp, _vp,
                           _vp, _vp, _vp, _vp, _vp],
    "vlj_debug_set_tiles": [_vp, C.c_int],
    "vlj_debug_set_step_threads": [_vp, C.c_uint32],
    "vlj_debug_set_step_lanes": [_vp, C.c_uint32],
    "vlj_debug_tile_info": [_vp, _P(C.c_uint32), _P(C.c_uint32), _P(C.c_uint32), _P(C.c_uint32)],
    "vlj_debug_read_tile_lists": [_vp, _vp],
}


def load(path=None):
    """Load the CUDA library (VLJ_LIBRARY overrides the in-tree build, e.g.
    for a tuning variant); raises if it has not been built."""
    path = path or os.environ.get("VLJ_LIBRARY") or LIB_PATH
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build the CUDA library first (python virial-engine_b200/build.py)")
    lib = C.CDLL(path)
    for name, args in SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = _st
    lib.vlj_last_error.restype = C.c_char_p
    lib.vlj_last_error.argtypes = []
    lib.vlj_status_name.restype = C.c_char_p
    lib.vlj_status_name.argtypes = [C.c_int]
    return lib


def ptr(a):
    """Address of a numpy array's data."""
    return a.ctypes.data_as(C.c_void_p)
