"""ctypes binding of libdsmc_b200.so (the C ABI declared in include/dsmc_b200.h).

The library is loaded from this package directory; a missing library is an
error, never a silent fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libdsmc_b200.so"

DSMC_OK = 0
DSMC_ERR_ARG = 1
DSMC_ERR_IO = 2
DSMC_ERR_CUDA = 3
DSMC_ERR_CAPACITY = 4
DSMC_ERR_CONFIG = 5
DSMC_ERR_STATE = 6
DSMC_ERR_NOT_FOUND = 7
DSMC_ERR_NO_DEVICE = 8

# error bits of dsmc_device_status (include/dsmc_b200.h)
EBIT_CELL, EBIT_FACET, EBIT_RESEED, EBIT_SPILL_FULL, EBIT_SMEM, EBIT_NAN, EBIT_STRANDED, EBIT_WALL = (
    1, 2, 4, 8, 16, 32, 64, 512)
EBIT_FATAL = EBIT_CELL | EBIT_RESEED | EBIT_SPILL_FULL | EBIT_SMEM | EBIT_NAN | EBIT_WALL

PREC_SPLIT32 = 0
PREC_FP64 = 1

# every entry point declared in include/dsmc_b200.h
EXPORTED = [
    "dsmc_settings_defaults", "dsmc_settings_load_ini", "dsmc_world_read_header", "dsmc_world_read",
    "dsmc_world_write", "dsmc_geometry_packed_spheres", "dsmc_geometry_finish", "dsmc_geometry_finish_gpu",
    "dsmc_ctx_create", "dsmc_ctx_destroy", "dsmc_last_error", "dsmc_sync", "dsmc_system_add",
    "dsmc_system_add_world", "dsmc_system_info_get", "dsmc_particles_init", "dsmc_particles_set",
    "dsmc_particles_count", "dsmc_particles_get", "dsmc_step", "dsmc_stage_move", "dsmc_stage_sort",
    "dsmc_stage_collide", "dsmc_stage_sample", "dsmc_tallies_get", "dsmc_tallies_reset", "dsmc_cells_get",
    "dsmc_cells_set_state", "dsmc_device_status", "dsmc_stream", "dsmc_counters_get", "dsmc_cells_layout",
    "dsmc_ctx_set_capacity", "dsmc_pass_info", "dsmc_geometry_finish_gpu_noalloc", "dsmc_ctx_set_timing",
    "dsmc_pass_times_get", "dsmc_state_file_read", "dsmc_state_file_write", "dsmc_tocontinue_read",
    "dsmc_tocontinue_write", "dsmc_continue_from", "dsmc_checkpoint_save", "dsmc_checkpoint_load",
    "dsmc_profile_sums_get", "dsmc_profiles_finish", "dsmc_profiles_get", "dsmc_measures_get",
    "dsmc_system_add_slab", "dsmc_exchange_take", "dsmc_exchange_put", "dsmc_particles_init_field",
    "dsmc_field_accumulate", "dsmc_tuning_set", "dsmc_tuning_get", "dsmc_particles_init_many",
    "dsmc_particles_init_field_many",
]
# every entry point declared in include/dsmc_surrogate.h
EXPORTED_SURROGATE = [
    "dsmc_sg_conv3", "dsmc_sg_conv3_wgrad", "dsmc_sg_bias_grad", "dsmc_sg_pool2", "dsmc_sg_pool2_bwd",
    "dsmc_sg_up2", "dsmc_sg_up2_bwd", "dsmc_sg_pack_input", "dsmc_sg_head", "dsmc_sg_loss_head_bwd",
    "dsmc_sg_adam", "dsmc_sg_pack_weights", "dsmc_sg_status", "dsmc_sg_sample_flux_loss",
]


class Tuning(C.Structure):
    """Mirror of dsmc_tuning: launch shape of the production pass."""
    _fields_ = [("blocks_per_sm", C.c_int * 5), ("ring", C.c_int), ("collide_claim", C.c_int)]


class DsmcError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"dsmc error {code}: {msg}")
        self.code = code


class Settings(C.Structure):
    """Mirror of dsmc_settings (the reference's Settings, dsmc/settings.h:11-49)."""
    _fields_ = [
        ("timesteps", C.c_int), ("statistics_interval", C.c_int), ("atoms_per_molecule", C.c_int),
        ("cells_x", C.c_int), ("cells_y", C.c_int), ("cells_z", C.c_int), ("flow_direction", C.c_int),
        ("sampling_bins", C.c_int), ("seed", C.c_int), ("max_molecules_per_node", C.c_int),
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("mass", C.c_double), ("temperature", C.c_double), ("wall_temperature", C.c_double),
        ("gravity", C.c_double), ("density", C.c_double), ("diam", C.c_double),
        ("Lx", C.c_double), ("Ly", C.c_double), ("Lz", C.c_double), ("dt", C.c_double),
        ("alpha_n", C.c_double), ("alpha_t", C.c_double), ("viscosity", C.c_double),
        ("surface_model", C.c_int), ("sample_begin", C.c_int), ("rng_seed", C.c_uint64),
        ("world", C.c_char * 512), ("load_previous_state", C.c_int),
    ]


class WorldHeader(C.Structure):
    _fields_ = [("porosity_global", C.c_float), ("porosity", C.c_float),
                ("global_nx", C.c_uint32), ("global_ny", C.c_uint32), ("global_nz", C.c_uint32),
                ("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32)]


class SphereParams(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("radius", C.c_double),
                ("spheres_type", C.c_int), ("spheres_num", C.c_int), ("wanted_porosity", C.c_double),
                ("seed", C.c_int), ("inverted", C.c_int), ("prevent_overlap", C.c_int),
                ("number_of_neighbor_averages", C.c_int)]


class SystemInfo(C.Structure):
    _fields_ = [("num_particles", C.c_int64), ("num_cells_total", C.c_int), ("num_active_cells", C.c_int),
                ("volume", C.c_double), ("porosity", C.c_double), ("atoms_per_molecule", C.c_double),
                ("dt", C.c_double), ("expected_particles", C.c_int64), ("slots", C.c_int),
                ("volume_global", C.c_double)]


class Tallies(C.Structure):
    _fields_ = [("step", C.c_uint64), ("collisions", C.c_uint64), ("wall_collisions", C.c_uint64),
                ("reseeds", C.c_uint64), ("particle_steps", C.c_uint64), ("count_periodic", C.c_int64 * 3),
                ("samples", C.c_uint64), ("candidates", C.c_uint64), ("kinetic_energy", C.c_double),
                ("temperature", C.c_double), ("flux", C.c_double), ("time", C.c_double), ("stranded", C.c_uint64)]


class Measures(C.Structure):
    _fields_ = [("step", C.c_uint64), ("t_ns", C.c_double), ("energy_eV", C.c_double),
                ("temperature_K", C.c_double), ("number_flow_rate", C.c_double),
                ("volumetric_flow_rate", C.c_double), ("pressure_Pa", C.c_double),
                ("permeability_darcy", C.c_double), ("collisions", C.c_uint64), ("wall_collisions", C.c_uint64),
                ("molecules", C.c_uint64)]


_lib = None

_P = C.c_void_p
_D = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)
_U8 = C.POINTER(C.c_uint8)
_I32 = C.POINTER(C.c_int32)


def load() -> C.CDLL:
    """Loads the in-tree library (built by master_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run master_b200.build.build() first")
    lib = C.CDLL(str(LIB_PATH))
    sig = {
        "dsmc_settings_defaults": [C.POINTER(Settings)],
        "dsmc_settings_load_ini": [C.c_char_p, C.POINTER(Settings)],
        "dsmc_world_read_header": [C.c_char_p, C.POINTER(WorldHeader)],
        "dsmc_world_read": [C.c_char_p, _U8, _F, _F, _F],
        "dsmc_world_write": [C.c_char_p, C.c_uint32, C.c_uint32, C.c_uint32, _U8, _F, _F, _F, C.c_int, C.c_int,
                             C.c_int],
        "dsmc_geometry_packed_spheres": [C.POINTER(SphereParams), _U8, _F, _F, _F, _F],
        "dsmc_geometry_finish": [C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, _U8, _F, _F, _F],
        "dsmc_geometry_finish_gpu": [C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, _U8, _F, _F, _F],
        "dsmc_geometry_finish_gpu_noalloc": [C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, _U8, _F, _F,
                                             _F],
        "dsmc_ctx_create": [C.c_int, C.c_int, C.POINTER(_P)],
        "dsmc_ctx_destroy": [_P],
        "dsmc_last_error": [_P],
        "dsmc_sync": [_P],
        "dsmc_system_add": [_P, C.POINTER(Settings), C.c_uint32, C.c_uint32, C.c_uint32, _U8, _F, _F, _F, C.c_float,
                            C.POINTER(C.c_int)],
        "dsmc_system_add_world": [_P, C.POINTER(Settings), C.POINTER(C.c_int)],
        "dsmc_system_info_get": [_P, C.c_int, C.POINTER(SystemInfo)],
        "dsmc_particles_init": [_P, C.c_int, C.c_int64],
        "dsmc_particles_set": [_P, C.c_int, C.c_int64, _D, _D],
        "dsmc_particles_count": [_P, C.c_int, C.POINTER(C.c_int64)],
        "dsmc_particles_get": [_P, C.c_int, C.c_int64, _D, _D, _I32, C.POINTER(C.c_int64)],
        "dsmc_step": [_P, C.c_int],
        "dsmc_stage_move": [_P],
        "dsmc_stage_sort": [_P],
        "dsmc_stage_collide": [_P],
        "dsmc_stage_sample": [_P],
        "dsmc_tallies_get": [_P, C.c_int, C.POINTER(Tallies)],
        "dsmc_tallies_reset": [_P, C.c_int],
        "dsmc_cells_get": [_P, C.c_int, C.c_int, _I32, _I32, _D, _D, _D, _D, C.POINTER(C.c_int)],
        "dsmc_cells_set_state": [_P, C.c_int, _D, _D],
        "dsmc_device_status": [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)],
        "dsmc_stream": [_P],
        "dsmc_counters_get": [_P, C.c_int, C.POINTER(C.c_int64)],
        "dsmc_ctx_set_capacity": [_P, C.c_double, C.c_int],
        "dsmc_pass_info": [_P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)],
        "dsmc_ctx_set_timing": [_P, C.c_int],
        "dsmc_pass_times_get": [_P, _D, C.POINTER(C.c_int64)],
        "dsmc_state_file_read": [C.c_char_p, C.c_int64, _D, _D, C.POINTER(C.c_int64)],
        "dsmc_state_file_write": [C.c_char_p, C.c_int64, _D, _D],
        "dsmc_tocontinue_read": [C.c_char_p, _D, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                 C.POINTER(C.c_uint64)],
        "dsmc_tocontinue_write": [C.c_char_p, C.c_double, C.c_uint64, C.c_uint64, C.c_uint64],
        "dsmc_continue_from": [_P, C.c_int, C.c_double, C.c_uint64, C.c_uint64, C.c_uint64],
        "dsmc_checkpoint_save": [_P, C.c_char_p],
        "dsmc_checkpoint_load": [_P, C.c_char_p],
        "dsmc_profile_sums_get": [_P, C.c_int, C.c_int, _D, C.POINTER(C.c_int)],
        "dsmc_measures_get": [_P, C.c_int, C.POINTER(Measures)],
        "dsmc_system_add_slab": [_P, C.POINTER(Settings), C.c_uint32, C.c_uint32, C.c_uint32, _U8, _F, _F, _F,
                                 C.c_float, C.c_int, C.c_int, C.POINTER(C.c_int)],
        "dsmc_exchange_take": [_P, C.c_int64, C.c_void_p, C.c_int, C.POINTER(C.c_int64)],
        "dsmc_exchange_put": [_P, C.c_int, C.c_int64, C.c_void_p, C.c_int],
        "dsmc_particles_init_field": [_P, C.c_int, C.c_int64, C.c_void_p, C.c_void_p, C.c_int],
        "dsmc_particles_init_many": [_P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int64)],
        "dsmc_particles_init_field_many": [_P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int64),
                                           C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_int],
        "dsmc_field_accumulate": [_P, C.c_int, C.c_void_p, C.c_int],
        "dsmc_tuning_set": [_P, C.POINTER(Tuning)],
        "dsmc_tuning_get": [_P, C.POINTER(Tuning), C.POINTER(Tuning)],
        "dsmc_profiles_finish": [C.POINTER(Settings), C.c_double, C.c_int, _D, _D, _D, _D, _D, _D, _D],
        "dsmc_profiles_get": [_P, C.c_int, C.c_int, _D, _D, _D, _D, _D, _D, C.POINTER(C.c_int)],
        "dsmc_cells_layout": [C.POINTER(Settings), C.c_uint32, C.c_uint32, C.c_uint32, _U8, C.c_int, _I32, _I32,
                              _I32, _D, _D, C.POINTER(C.c_int)],
    }
    V, I = C.c_void_p, C.c_int
    sig.update({
        "dsmc_sg_conv3": [V, I, I, V, I, I, I, V, V, I, V, I, I, I, V, I, I],
        "dsmc_sg_conv3_wgrad": [V, I, I, V, I, I, I, V, I, I, I, V],
        "dsmc_sg_bias_grad": [V, I, I, V, I, I, I, V],
        "dsmc_sg_pool2": [V, I, I, V, I, I, I, V, I, I],
        "dsmc_sg_pool2_bwd": [V, I, I, V, I, I, V, I, I, V, I, I, I, V, I, I],
        "dsmc_sg_up2": [V, I, I, V, I, I, I, V, I, I],
        "dsmc_sg_up2_bwd": [V, I, I, V, I, I, V, I, I, I, V, I, I],
        "dsmc_sg_pack_input": [V, I, I, V, V, V],
        "dsmc_sg_head": [V, I, I, V, I, I, V, V, V],
        "dsmc_sg_loss_head_bwd": [V, I, I, V, V, V, V, C.c_float, V, I, I, V, V, V, V, I, I, V, V, I],
        "dsmc_sg_sample_flux_loss": [V, I, I, V, V, V, I, C.c_float, V, V, V],
        "dsmc_sg_adam": [V, V, V, V, V, C.c_int64, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int64],
        "dsmc_sg_pack_weights": [V, V, I, I, V, V],
        "dsmc_sg_status": [C.POINTER(C.c_uint), I],
    })
    for name, args in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = C.c_int
    lib.dsmc_ctx_destroy.restype = None
    lib.dsmc_last_error.restype = C.c_char_p
    lib.dsmc_stream.restype = C.c_void_p
    _lib = lib
    return lib


def ptr(a: np.ndarray | None, ctype):
    if a is None:
        return C.cast(None, C.POINTER(ctype))
    assert a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(ctype))


def check(rc: int, ctx=None) -> None:
    if rc != DSMC_OK:
        msg = load().dsmc_last_error(ctx)
        raise DsmcError(rc, msg.decode() if msg else "")
