"""ctypes binding of the C-ABI in include/felbm_b200.h.

Loads felbm_gpu_b200/_lib/libfelbm_b200.so (built in-tree by
``make -C felbm_gpu_b200`` or ``__graft_entry__.build()``), or the build named
by the environment variable FELBM_B200_LIB. There is no fallback: if the
library is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os

from ._abi import *  # noqa: F401,F403  (structure layouts and constants)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("FELBM_B200_LIB") or os.path.join(_HERE, "_lib", "libfelbm_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"felbm_gpu_b200: native library not built ({LIB_PATH}); run `make -C felbm_gpu_b200`"
    )
lib = C.CDLL(LIB_PATH)

_dp = C.POINTER(C.c_double)
_vp = C.c_void_p
_i64p = C.POINTER(C.c_int64)
_u8p = C.POINTER(C.c_uint8)
_i32p = C.POINTER(C.c_int32)
_fp = C.POINTER(C.c_float)

# name -> (restype, argtypes); every symbol declared in include/felbm_b200.h
SIGNATURES = {
    "fe_params_default": (C.c_int, [C.POINTER(FeParams)]),
    "fe_params_derive": (C.c_int, [C.POINTER(FeParams)]),
    "fe_driver_cfg_default": (C.c_int, [C.POINTER(FeDriverCfg)]),
    "fe_cfg_read": (C.c_int, [C.c_char_p, C.POINTER(FeParams), C.POINTER(FeOpenBnd), C.POINTER(FeDriverCfg)]),
    "fe_cfg_switch_log": (C.c_int, [C.POINTER(FeParams), C.c_char_p, C.c_int]),
    "fe_engine_create": (C.c_int, [C.POINTER(FeParams), C.c_int, C.c_int, C.c_int, _u8p, C.c_int, C.POINTER(_vp)]),
    "fe_engine_destroy": (C.c_int, [_vp]),
    "fe_engine_size": (C.c_int, [_vp, _i64p, _i64p]),
    "fe_set_params": (C.c_int, [_vp, C.POINTER(FeParams)]),
    "fe_engine_stream": (C.c_void_p, [_vp]),
    "fe_upload_state": (C.c_int, [_vp, _dp, _dp, C.c_int64]),
    "fe_upload_equilibrium": (C.c_int, [_vp, _dp, _dp, C.c_double, C.c_int64]),
    "fe_download_state": (C.c_int, [_vp, _dp, _dp, C.c_int64]),
    "fe_set_open_bnd": (C.c_int, [_vp, C.POINTER(FeOpenBnd)]),
    "fe_step": (C.c_int, [_vp, C.c_int]),
    "fe_apply_mass_correction": (C.c_int, [_vp, _dp]),
    "fe_run": (C.c_int, [_vp, C.c_int]),
    "fe_set_time": (C.c_int, [_vp, C.c_int64]),
    "fe_get_time": (C.c_int, [_vp, _i64p]),
    "fe_set_forcing_factor": (C.c_int, [_vp, C.c_double]),
    "fe_record_target_mass": (C.c_int, [_vp]),
    "fe_set_target_mass": (C.c_int, [_vp, C.c_double]),
    "fe_get_target_mass": (C.c_int, [_vp, _dp]),
    "fe_current_mass": (C.c_int, [_vp, _dp]),
    "fe_download_fields": (C.c_int, [_vp, C.POINTER(FeFields)]),
    "fe_flow_stats": (C.c_int, [_vp, _dp]),
    "fe_flow_stats_launch": (C.c_int, [_vp]),
    "fe_flow_stats_ready": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "fe_flow_stats_collect": (C.c_int, [_vp, _dp]),
    "fe_mass_weight_noalloc": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]),
    "fe_time_run": (C.c_int, [_vp, C.c_int, _fp]),
    "fe_time_kernels": (C.c_int, [_vp, C.c_int, _fp, C.c_int]),
    "fe_launch_count": (C.c_int, [_vp, _i64p]),
    "fe_batch_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "fe_batch_destroy": (C.c_int, [_vp]),
    "fe_batch_add": (C.c_int, [_vp, _vp]),
    "fe_batch_remove": (C.c_int, [_vp, _vp]),
    "fe_batch_size": (C.c_int, [_vp, C.POINTER(C.c_int), _i64p]),
    "fe_batch_run": (C.c_int, [_vp, C.c_int]),
    "fe_batch_launch": (C.c_int, [_vp, C.c_int]),
    "fe_batch_wait": (C.c_int, [_vp]),
    "fe_batch_time_run": (C.c_int, [_vp, C.c_int, _fp]),
    "fe_batch_launch_count": (C.c_int, [_vp, _i64p]),
    "fe_tracers_create": (C.c_int, [_vp, C.POINTER(FeTracerConfig), C.c_int64, _dp, _dp, _i64p,
                                    C.POINTER(C.c_void_p)]),
    "fe_tracers_destroy": (C.c_int, [_vp]),
    "fe_tracers_step": (C.c_int, [_vp]),
    "fe_tracers_download": (C.c_int, [_vp, _dp, _dp]),
    "fe_tracers_stretch_rows": (C.c_int, [_vp, _dp, C.c_int64, _i64p]),
    "fe_tracers_stretch_state": (C.c_int, [_vp, _dp, _dp]),
    "fe_tracers_set_stretch_state": (C.c_int, [_vp, _dp, _dp]),
    "fe_tracers_set_velocity": (C.c_int, [_vp, _dp, _dp]),
    "fe_tracers_seed": (C.c_int, [_u8p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _dp, C.c_int, C.c_int64,
                                  C.c_uint64, _dp, _i32p]),
    "fe_write_fields_h5": (C.c_int, [_vp, C.c_char_p, C.c_int, C.c_int]),
    "fe_write_geometry_h5": (C.c_int, [C.c_char_p, _u8p, C.c_int, C.c_int, C.c_int]),
    "fe_checkpoint_write": (C.c_int, [_vp, C.c_char_p, C.c_uint32]),
    "fe_settle_mass_correction": (C.c_int, [_vp]),
    "fe_checkpoint_read": (C.c_int, [_vp, C.c_char_p, C.POINTER(C.c_uint32)]),
    "fe_write_particles_h5": (C.c_int, [C.c_char_p, C.c_int64, _dp, _dp, _i64p, _dp, _i32p, _dp, _dp]),
    "fe_geom_tiff_stack": (C.c_int, [C.POINTER(C.c_char_p), C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _u8p,
                                     C.c_int64]),
    "fe_autotune": (C.c_int, [C.POINTER(FeParams), C.c_int, C.c_int, C.c_int, _u8p, C.c_int, C.c_int,
                              C.POINTER(FeTuneReport)]),
    "fe_engine_layout": (C.c_int, [_vp, _i32p, _i32p]),
    "fe_tune_save": (C.c_int, [C.c_char_p]),
    "fe_tune_load": (C.c_int, [C.c_char_p]),
    "fe_tune_clear": (C.c_int, []),
    "fe_write_series": (C.c_int, [C.c_char_p, C.c_int, C.c_uint32, _dp, C.c_int64]),
    "fe_write_stretching": (C.c_int, [C.c_char_p, C.c_int, _dp, C.c_int64]),
    "fe_h5_write_dataset": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_int, _i64p, C.c_void_p, C.c_int]),
    "fe_h5_read_dataset": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(C.c_int), _i64p, C.POINTER(C.c_int),
                                     C.c_void_p, C.c_int64]),
    "fe_server_create": (C.c_int, [C.POINTER(FeServerConfig), C.POINTER(C.c_void_p)]),
    "fe_server_submit": (C.c_int, [_vp, C.POINTER(FeRequest)]),
    "fe_server_poll": (C.c_int, [_vp, C.POINTER(FeResult), C.c_int, C.POINTER(C.c_int)]),
    "fe_server_free_result": (C.c_int, [C.POINTER(FeResult)]),
    "fe_server_wait_idle": (C.c_int, [_vp, C.c_double]),
    "fe_server_get_stats": (C.c_int, [_vp, C.POINTER(FeServerStats)]),
    "fe_server_destroy": (C.c_int, [_vp]),
    "fe_last_error": (C.c_char_p, []),
    "fe_version": (C.c_char_p, []),
    "fe_geom_grf": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_uint64, C.c_int, C.c_int,
                              _u8p, _dp]),
    "fe_geom_cylinders": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                    C.c_uint64, C.c_int, _u8p, _dp]),
    "fe_geom_spheres": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_double, C.c_uint64, _u8p]),
    "fe_geom_pad_open": (C.c_int, [_u8p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.POINTER(C.c_int), _u8p]),
    "fe_geom_open_lists": (C.c_int, [_u8p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p,
                                     _i32p, _i32p, _i32p, _dp]),
    "fe_geom_sites": (C.c_int, [_u8p, C.c_int, C.c_int, C.c_int, _i64p, _i64p]),
    "fe_init_order_parameter": (C.c_int, [_u8p, C.c_int, C.c_int, C.c_int, C.c_int, _dp, C.c_double, _dp]),
    "fe_init_equilibrium": (C.c_int, [C.c_int64, _dp, _dp, _dp, _dp, _dp, C.c_double, C.c_double, _dp, _dp]),
}

for _name, (_res, _args) in SIGNATURES.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


class FeError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"felbm_b200 error {status}: {msg}")
        self.status = status


def check(status: int) -> None:
    if status != FE_OK:
        raise FeError(status, lib.fe_last_error().decode())
