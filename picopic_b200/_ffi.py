"""ctypes binding of libpcg.so (the C ABI in include/pcg.h).

The library is loaded from this package directory only; when it is missing
the import fails loudly, there is no other implementation to fall back to.
"""
from __future__ import annotations

import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libpcg.so")

PCG_OK = 0
STATUS = {0: "PCG_OK", -1: "PCG_ERR_ARG", -2: "PCG_ERR_CUDA", -3: "PCG_ERR_NOMEM",
          -4: "PCG_ERR_STATE", -5: "PCG_ERR_CAPACITY", -10: "PCG_ERR_NAN",
          -11: "PCG_ERR_SUPERLUMINAL", -12: "PCG_ERR_TIMEOUT", -13: "PCG_ERR_UNSUPPORTED"}


class PcgError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where}: {STATUS.get(code, code)}: {msg}")
        self.code = code


class Config(ctypes.Structure):
    _fields_ = [("nr", ctypes.c_int), ("nz", ctypes.c_int),
                ("radius", ctypes.c_double), ("longitude", ctypes.c_double),
                ("dt", ctypes.c_double), ("t_start", ctypes.c_double),
                ("pml_size", ctypes.c_int * 4), ("pml_sigma", ctypes.c_double * 2),
                ("pusher", ctypes.c_int), ("current", ctypes.c_int),
                ("precision", ctypes.c_int), ("quirks", ctypes.c_int),
                ("device", ctypes.c_int), ("seed", ctypes.c_uint64)]


class Diagnostics(ctypes.Structure):
    _fields_ = [("time", ctypes.c_double), ("steps", ctypes.c_uint64),
                ("particles", ctypes.c_uint64), ("removed", ctypes.c_uint64),
                ("move_errors", ctypes.c_uint64), ("particle_steps", ctypes.c_uint64),
                ("field_energy_e", ctypes.c_double), ("field_energy_h", ctypes.c_double),
                ("kinetic_energy", ctypes.c_double), ("kernel_launches", ctypes.c_uint64)]


class Band(ctypes.Structure):
    """pcg_band: one band of a device-to-device transfer."""
    _fields_ = [("slot", ctypes.c_int), ("lo", ctypes.c_double), ("hi", ctypes.c_double),
                ("shift", ctypes.c_double), ("dst", ctypes.c_void_p), ("dst_slot", ctypes.c_int),
                ("append", ctypes.c_int)]


_D = ctypes.c_double
_PD = ctypes.POINTER(ctypes.c_double)
_PF = ctypes.POINTER(ctypes.c_float)
_PI32 = ctypes.POINTER(ctypes.c_int32)
_H = ctypes.c_void_p

# name -> (restype, argtypes); every export of include/pcg.h
SIGNATURES = {
    "pcg_abi_version": (ctypes.c_int, []),
    "pcg_create": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(ctypes.c_void_p)]),
    "pcg_destroy": (ctypes.c_int, [_H]),
    "pcg_last_error": (ctypes.c_char_p, [_H]),
    "pcg_add_species": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_char_p, _D, _D, ctypes.c_size_t,
                                       ctypes.POINTER(ctypes.c_int)]),
    "pcg_add_beam": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_char_p, _D, _D, ctypes.c_size_t,
                                    ctypes.c_uint, _D, _D, _D, _D, _D, _D, _D,
                                    ctypes.POINTER(ctypes.c_int)]),
    "pcg_import_species": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_size_t] + [_PD] * 6),
    "pcg_append_species": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_size_t] + [_PD] * 6),
    "pcg_count": (ctypes.c_int, [_H, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]),
    "pcg_export_species": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_size_t] + [_PD] * 6 +
                           [_PI32, _PI32, ctypes.POINTER(ctypes.c_size_t)]),
    "pcg_set_field": (ctypes.c_int, [_H, ctypes.c_int, _PD]),
    "pcg_export_field": (ctypes.c_int, [_H, ctypes.c_int, _PD]),
    "pcg_get_field_columns": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, ctypes.c_int, _PD]),
    "pcg_set_field_columns": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, ctypes.c_int, _PD]),
    "pcg_export_species_range": (ctypes.c_int, [_H, ctypes.c_int, _D, _D, ctypes.c_size_t] + [_PD] * 6 +
                                 [ctypes.POINTER(ctypes.c_size_t)]),
    "pcg_keep_species_range": (ctypes.c_int, [_H, ctypes.c_int, _D, _D]),
    "pcg_transfer_species_range": (ctypes.c_int, [_H, ctypes.c_int, _D, _D, _D, _H, ctypes.c_int, ctypes.c_int,
                                                  ctypes.POINTER(ctypes.c_size_t)]),
    "pcg_transfer_species_bands": (ctypes.c_int, [_H, ctypes.c_int, ctypes.POINTER(Band),
                                                  ctypes.POINTER(ctypes.c_size_t)]),
    "pcg_copy_field_columns": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, ctypes.c_int, _H, ctypes.c_int]),
    "pcg_get_device": (ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_int)]),
    "pcg_stage": (ctypes.c_int, [_H, ctypes.c_int]),
    "pcg_step": (ctypes.c_int, [_H, ctypes.c_int]),
    "pcg_synchronize": (ctypes.c_int, [_H]),
    "pcg_diag": (ctypes.c_int, [_H, ctypes.POINTER(Diagnostics)]),
    "pcg_get_stream": (ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_void_p)]),
    "pcg_seed_plasma": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_size_t, _D, _D, ctypes.c_uint64]),
    "pcg_seed_plasma_cells": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_uint, _D, _D, _D, ctypes.c_uint64]),
    "pcg_set_beam_profile": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, _D, _D]),
    "pcg_enable_timers": (ctypes.c_int, [_H, ctypes.c_int]),
    "pcg_kernel_times": (ctypes.c_int, [_H, _PD, ctypes.POINTER(ctypes.c_int), ctypes.c_int]),
    "pcg_current_vb_f64_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _D, _D, _D,
                                                  ctypes.c_size_t, _D] + [ctypes.c_void_p] * 9 +
                                   [ctypes.c_int, ctypes.c_void_p,
                                    ctypes.POINTER(ctypes.c_ulonglong)]),
    "pcg_node_charge": (ctypes.c_int, [_H, _PD]),
    "pcg_divergence": (ctypes.c_int, [_H, ctypes.c_int, _PD]),
    "pcg_collide": (ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_ulonglong)]),
    "pcg_set_collision_model": (ctypes.c_int, [_H, _PF, _PF]),
    "pcg_collide_learned": (ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_ulonglong),
                                           ctypes.POINTER(ctypes.c_ulonglong)]),
    "pcg_cell_moments": (ctypes.c_int, [_H, _PD]),
    "pcg_set_collisions": (ctypes.c_int, [_H, ctypes.c_int]),
    "pcg_set_collision_scheme": (ctypes.c_int, [_H, ctypes.c_int]),
    "pcg_set_collision_crowding": (ctypes.c_int, [_H, ctypes.c_uint]),
    "pcg_step_status": (ctypes.c_int, [_H]),
    "pcg_set_external_fields": (ctypes.c_int, [_H, ctypes.c_char_p, _PD, ctypes.c_int, ctypes.c_char_p, _PD,
                                               ctypes.c_int]),
    "pcg_species_map": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, _PD]),
    "pcg_set_tiling": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "pcg_tile_sort": (ctypes.c_int, [_H, ctypes.c_int, ctypes.POINTER(ctypes.c_uint),
                                     ctypes.POINTER(ctypes.c_ulonglong)]),
    "pcg_ensemble_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_void_p)]),
    "pcg_ensemble_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]),
    "pcg_ensemble_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "pcg_ensemble_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "pcg_ensemble_set_graph": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "pcg_ensemble_graph_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_ulonglong),
                                               ctypes.POINTER(ctypes.c_float)]),
    "pcg_collide_expectation": (ctypes.c_int, [_H, _PD]),
    "pcg_cell_features": (ctypes.c_int, [_H, _PF, _PD]),
    "pcg_mlp_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)]),
    "pcg_mlp_destroy": (ctypes.c_int, [_H]),
    "pcg_mlp_get_params": (ctypes.c_int, [_H, _PF]),
    "pcg_mlp_set_params": (ctypes.c_int, [_H, _PF]),
    "pcg_mlp_forward": (ctypes.c_int, [_H, _PF, ctypes.c_size_t, _PF]),
    "pcg_mlp_forward_tc": (ctypes.c_int, [_H, _PF, ctypes.c_size_t, _PF, _PF]),
    "pcg_mlp_gradient": (ctypes.c_int, [_H, _PF, _PF, ctypes.c_size_t, _PF, _PF]),
    "pcg_mlp_set_data": (ctypes.c_int, [_H, _PF, _PF, ctypes.c_size_t]),
    "pcg_mlp_train": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, ctypes.c_float, _PF]),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load libpcg.so and declare every exported function."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m picopic_b200.build`")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.pcg_abi_version() != 1:
        raise ImportError("libpcg.so ABI version mismatch")
    _lib = lib
    return lib
