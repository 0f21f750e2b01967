"""ctypes binding of libpsl_b200.so (the C ABI declared in include/psl.h).

There is no fallback: if the library is missing or a call fails, an exception is raised.
"""
from __future__ import annotations

import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libpsl_b200.so")

PSL_OK = 0
STORAGE = {"f32": 0, "f16": 1, "bf16": 2, "f64": 3}
STORAGE_BYTES = {0: 4, 1: 2, 2: 2, 3: 8}

CELL_SKIP, CELL_FLUID, CELL_SOLID, CELL_GIVEN_U, CELL_GIVEN_RHO, CELL_GIVEN_NONE, CELL_GIVEN_BOTH, CELL_MIRROR = range(8)


class PslInfo(ctypes.Structure):
    _fields_ = [
        ("grid_id", ctypes.c_int),
        ("res", ctypes.c_float),
        ("cell_count_x", ctypes.c_int), ("cell_count_y", ctypes.c_int), ("cell_count_z", ctypes.c_int),
        ("ox", ctypes.c_float), ("oy", ctypes.c_float), ("oz", ctypes.c_float),
        ("nu", ctypes.c_float),
        ("dt_phys", ctypes.c_float),
        ("i_subgrid_start", ctypes.c_int), ("j_subgrid_start", ctypes.c_int), ("k_subgrid_start", ctypes.c_int),
        ("i_subgrid_end", ctypes.c_int), ("j_subgrid_end", ctypes.c_int), ("k_subgrid_end", ctypes.c_int),
    ]


class PslSphereCase(ctypes.Structure):
    _fields_ = [
        ("sphere_x", ctypes.c_float), ("sphere_y", ctypes.c_float), ("sphere_z", ctypes.c_float),
        ("sphere_r", ctypes.c_float),
        ("u_in", ctypes.c_float),
        ("rho_given", ctypes.c_float),
        ("wall_mode", ctypes.c_int),
        ("smagorinsky", ctypes.c_float),
        ("seed", ctypes.c_uint32),
        ("noise_amp", ctypes.c_float),
    ]


class PslBatchTuning(ctypes.Structure):
    _fields_ = [
        ("threads", ctypes.c_int),
        ("tile_cells", ctypes.c_int),
        ("blocks_per_sm", ctypes.c_int),
        ("ms_per_step", ctypes.c_float),
    ]


class PslSgsMlp(ctypes.Structure):
    _fields_ = [
        ("w1", (ctypes.c_float * 10) * 32),
        ("b1", ctypes.c_float * 32),
        ("w2", (ctypes.c_float * 32) * 32),
        ("b2", ctypes.c_float * 32),
        ("w3", ctypes.c_float * 32),
        ("b3", ctypes.c_float),
        ("in_shift", ctypes.c_float * 10),
        ("in_scale", ctypes.c_float * 10),
        ("out_scale", ctypes.c_float),
    ]


class PslFlowReport(ctypes.Structure):
    _fields_ = [("ux", ctypes.c_double), ("uy", ctypes.c_double), ("uz", ctypes.c_double), ("rho", ctypes.c_double),
                ("area", ctypes.c_double)]


class PslError(RuntimeError):
    pass


_lib = None

# name -> (restype, argtypes); every entry point of include/psl.h
_SIGNATURES = {
    "psl_grid_create": (ctypes.c_int, [ctypes.POINTER(PslInfo), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "psl_grid_create_ex": (ctypes.c_int, [ctypes.POINTER(PslInfo), ctypes.c_int, ctypes.c_uint,
                                          ctypes.POINTER(ctypes.c_void_p)]),
    "psl_grid_get_layout": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                           ctypes.POINTER(ctypes.c_longlong)]),
    "psl_grid_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "psl_grid_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "psl_grid_get_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(PslInfo), ctypes.POINTER(ctypes.c_longlong),
                                         ctypes.POINTER(ctypes.c_int)]),
    "psl_apply_sphere_case": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(PslSphereCase)]),
    "psl_set_markers": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "psl_get_markers": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "psl_set_given": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float]),
    "psl_set_given_field": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "psl_set_smagorinsky": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_float]),
    "psl_set_smagorinsky_field": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "psl_forcing_torque": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_void_p,
                                          ctypes.c_void_p]),
    "psl_fill_equilibrium_sphere": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(PslSphereCase)]),
    "psl_fill_equilibrium_uniform": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                                    ctypes.c_float]),
    "psl_apply_streaming": (ctypes.c_int, [ctypes.c_void_p]),
    "psl_apply_local_cell_update": (ctypes.c_int, [ctypes.c_void_p]),
    "psl_apply_bc_periodic_x": (ctypes.c_int, [ctypes.c_void_p]),
    "psl_apply_bc_periodic_y": (ctypes.c_int, [ctypes.c_void_p]),
    "psl_apply_coarse_fine_grid_communication": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "psl_fill_coarse_grid_from_fine": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "psl_update_grid": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int]),
    "psl_sphere_force": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(PslSphereCase), ctypes.c_void_p]),
    "psl_sphere_force_async": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(PslSphereCase), ctypes.c_void_p]),
    "psl_momentum_exchange_force_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p,
                                                           ctypes.c_longlong, ctypes.c_void_p, ctypes.c_int,
                                                           ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                                           ctypes.c_void_p, ctypes.c_void_p]),
    "psl_get_populations": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "psl_get_macroscopic": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "psl_set_sgs_mlp": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(PslSgsMlp), ctypes.c_float]),
    "psl_set_sgs_mlp_interval": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "psl_sgs_mlp_infer": (ctypes.c_int, [ctypes.POINTER(PslSgsMlp), ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "psl_fill_equilibrium_field": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "psl_sgs_trainer_create": (ctypes.c_int, [ctypes.c_longlong, ctypes.POINTER(ctypes.c_void_p)]),
    "psl_sgs_trainer_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "psl_sgs_trainer_clear": (ctypes.c_int, [ctypes.c_void_p]),
    "psl_sgs_trainer_count": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]),
    "psl_sgs_trainer_add_samples": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong]),
    "psl_sgs_trainer_add_filtered": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                                    ctypes.c_uint]),
    "psl_sgs_trainer_get_samples": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_longlong,
                                                   ctypes.c_void_p, ctypes.c_void_p]),
    "psl_sgs_trainer_set_params": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(PslSgsMlp)]),
    "psl_sgs_trainer_get_params": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(PslSgsMlp)]),
    "psl_sgs_trainer_gradient": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_longlong,
                                                ctypes.POINTER(PslSgsMlp), ctypes.POINTER(ctypes.c_double)]),
    "psl_sgs_trainer_train": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_uint,
                                             ctypes.POINTER(ctypes.c_double)]),
    "psl_torque": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_void_p]),
    "psl_get_flow_report": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_void_p, ctypes.POINTER(PslFlowReport)]),
    "psl_set_body_force": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_float, ctypes.c_float, ctypes.c_float]),
    "psl_export_section_cut": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                              ctypes.c_float, ctypes.c_void_p, ctypes.c_longlong,
                                              ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "psl_enable_scalar_transport": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_float]),
    "psl_set_scalar_given_field": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "psl_get_scalar_populations": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "psl_set_scalar_populations": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "psl_get_scalar": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "psl_batch_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "psl_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "psl_batch_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "psl_batch_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "psl_batch_get_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "psl_batch_get_tuning": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(PslBatchTuning)]),
    "psl_batch_set_tuning": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(PslBatchTuning)]),
    "psl_batch_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(PslBatchTuning)]),
    "psl_set_populations": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "psl_get_shifts": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "psl_set_shifts": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "psl_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "psl_check_health": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "psl_debug_cells": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "psl_last_error": (ctypes.c_char_p, []),
    "psl_version": (ctypes.c_char_p, []),
}


def lib():
    """Load libpsl_b200.so (once).  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built: run `python -m periodicshiftlbm_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int, what: str = ""):
    if rc != PSL_OK:
        msg = lib().psl_last_error().decode(errors="replace")
        raise PslError(f"{what}: status {rc}: {msg}")


def call(name: str, *args):
    rc = getattr(lib(), name)(*args)
    check(rc, name)
    return rc
