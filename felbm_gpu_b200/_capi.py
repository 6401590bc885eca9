"""ctypes binding of the C-ABI in include/felbm_b200.h.

Loads felbm_gpu_b200/_lib/libfelbm_b200.so (built in-tree by
``make -C felbm_gpu_b200`` or ``__graft_entry__.build()``). There is no
fallback: if the library is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libfelbm_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"felbm_gpu_b200: native library not built ({LIB_PATH}); run `make -C felbm_gpu_b200`"
    )
lib = C.CDLL(LIB_PATH)

FE_OK, FE_ERR_ARG, FE_ERR_CUDA, FE_ERR_NO_DEVICE, FE_ERR_MEMORY, FE_ERR_STATE, FE_ERR_IO, FE_ERR_DIVERGED = range(8)
FE_F64, FE_F32, FE_F16S, FE_BF16S, FE_F16G, FE_BF16G = range(6)
FE_MRT_E, FE_MRT_EPS, FE_MRT_Q, FE_MRT_NU, FE_MRT_PI, FE_MRT_M = range(1, 7)
FE_RATE_S0, FE_RATE_MAGIC, FE_RATE_FIXED = range(3)
STORAGE = {"f64": FE_F64, "f32": FE_F32, "f16s": FE_F16S, "bf16s": FE_BF16S, "f16g": FE_F16G, "bf16g": FE_BF16G}


class FeParams(C.Structure):
    _fields_ = [
        ("rho0", C.c_double), ("rho1", C.c_double),
        ("tau0", C.c_double), ("tau1", C.c_double),
        ("interface_width", C.c_double), ("surface_tension", C.c_double),
        ("mobility_coeff", C.c_double), ("phi", C.c_double),
        ("kappa", C.c_double), ("beta", C.c_double), ("mobility", C.c_double), ("bnd_coeff", C.c_double),
        ("gx", C.c_double), ("gy", C.c_double), ("gz", C.c_double),
        ("fx", C.c_double), ("fy", C.c_double), ("fz", C.c_double),
        ("forcing_timedep", C.c_int), ("forcing_period", C.c_double),
        ("use_mrt", C.c_int), ("mrt_lambda", C.c_double),
        ("mrt_rate_mode", C.c_int * 7), ("mrt_rate_value", C.c_double * 7),
        ("use_halfway_bb", C.c_int), ("correct_op_mass", C.c_int),
        ("stream_matrix_free", C.c_int), ("grad_matrix_free", C.c_int),
        ("fused", C.c_int), ("fuse_collision", C.c_int),
        ("mrt_fast_transform", C.c_int), ("stream_inplace", C.c_int),
        ("storage", C.c_int),
        ("c_ref", C.c_double), ("p_ref", C.c_double),
        ("brick", C.c_int), ("graph_steps", C.c_int),
    ]


class FeOpenBnd(C.Structure):
    _fields_ = [
        ("n_inlet", C.c_int), ("inlet", C.POINTER(C.c_int32)), ("inlet_coord", C.POINTER(C.c_double)),
        ("n_outlet", C.c_int), ("outlet", C.POINTER(C.c_int32)),
        ("n_buf", C.c_int), ("buf_verts", C.POINTER(C.c_int32)), ("buf_refs", C.POINTER(C.c_int32)),
        ("copy_to_buffers", C.c_int),
        ("use_in_vel", C.c_int), ("use_in_prs", C.c_int), ("use_in_fluid", C.c_int),
        ("use_out_prs", C.c_int), ("use_out_fluid", C.c_int),
        ("u_in_x", C.c_double), ("u_in_y", C.c_double), ("u_in_z", C.c_double),
        ("p_in", C.c_double), ("p_out", C.c_double),
        ("c_out_fixed", C.c_double), ("rho_out_fixed", C.c_double),
        ("inlet_c_a", C.c_double),
        ("inlet_mode", C.c_int), ("split_axis", C.c_int),
        ("inlet_period", C.c_double), ("inlet_duty", C.c_double),
        ("inlet_ramp", C.c_double), ("split_pos", C.c_double),
    ]


_dp = C.POINTER(C.c_double)


class FeFields(C.Structure):
    _fields_ = [("rho", _dp), ("c", _dp), ("ux", _dp), ("uy", _dp), ("uz", _dp), ("p", _dp), ("mu", _dp)]


class FeTuneReport(C.Structure):
    _fields_ = [("brick", C.c_int), ("graph_steps", C.c_int), ("ncand", C.c_int), ("cand_brick", C.c_int * 8),
                ("cand_graph_steps", C.c_int * 8), ("cand_mlups", C.c_double * 8)]


BRICK = {"auto": 0, "8x8x8": 1, "16x16x1": 2, "8x8x4": 3, "16x8x8": 4}


class FeTracerConfig(C.Structure):
    _fields_ = [("substeps", C.c_int), ("order", C.c_int), ("velocity_skip", C.c_int), ("seed", C.c_uint64),
                ("stretching", C.c_int), ("phase_split", C.c_int), ("stretching_seed", C.c_uint64)]


class FeServerConfig(C.Structure):
    _fields_ = [("device", C.c_int), ("max_active", C.c_int), ("hbm_reserve_frac", C.c_double),
                ("chunk_steps", C.c_int), ("storage", C.c_int), ("fill_sites", C.c_int64)]


class FeRequest(C.Structure):
    _fields_ = [("id", C.c_int64), ("params", FeParams), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("solid", C.POINTER(C.c_uint8)), ("h0", C.POINTER(C.c_double)), ("g0", C.POINTER(C.c_double)),
                ("init_kind", C.c_int), ("init_a", C.c_double * 5), ("init_width", C.c_double),
                ("init_p", C.c_double), ("steps", C.c_int64), ("conv_tol", C.c_double),
                ("want_fields", C.c_int)]


class FeResult(C.Structure):
    _fields_ = [("id", C.c_int64), ("status", C.c_int), ("message", C.c_char * 160),
                ("sites", C.c_int64), ("steps_done", C.c_int64),
                ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double),
                ("mass0", C.c_double), ("mass_final", C.c_double), ("stats", C.c_double * 6),
                ("rho", C.POINTER(C.c_double)), ("c", C.POINTER(C.c_double)), ("ux", C.POINTER(C.c_double)),
                ("uy", C.POINTER(C.c_double)), ("uz", C.POINTER(C.c_double)), ("p", C.POINTER(C.c_double))]


class FeServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("admitted", C.c_int64), ("completed", C.c_int64),
                ("queued", C.c_int64), ("active", C.c_int64), ("peak_active", C.c_int64),
                ("site_steps", C.c_int64), ("busy_seconds", C.c_double), ("elapsed_seconds", C.c_double),
                ("mlups_busy", C.c_double), ("mlups_wall", C.c_double),
                ("ttr_p50", C.c_double), ("ttr_p99", C.c_double), ("ttr_max", C.c_double)]


_vp = C.c_void_p
_i64p = C.POINTER(C.c_int64)
_u8p = C.POINTER(C.c_uint8)
_i32p = C.POINTER(C.c_int32)
_fp = C.POINTER(C.c_float)

# name -> (restype, argtypes); every symbol declared in include/felbm_b200.h
SIGNATURES = {
    "fe_params_default": (C.c_int, [C.POINTER(FeParams)]),
    "fe_params_derive": (C.c_int, [C.POINTER(FeParams)]),
    "fe_engine_create": (C.c_int, [C.POINTER(FeParams), C.c_int, C.c_int, C.c_int, _u8p, C.c_int, C.POINTER(_vp)]),
    "fe_engine_destroy": (C.c_int, [_vp]),
    "fe_engine_size": (C.c_int, [_vp, _i64p, _i64p]),
    "fe_set_params": (C.c_int, [_vp, C.POINTER(FeParams)]),
    "fe_engine_stream": (C.c_void_p, [_vp]),
    "fe_upload_state": (C.c_int, [_vp, _dp, _dp, C.c_int64]),
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
    "fe_write_fields_h5": (C.c_int, [_vp, C.c_char_p, C.c_int]),
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
