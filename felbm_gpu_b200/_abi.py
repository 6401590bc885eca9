"""Structure layouts and constants of the C-ABI in include/felbm_b200.h, as
ctypes types. Loading this module loads no library: the CPU oracle's
wrappers (test infrastructure) share these layouts without the engine.
"""
from __future__ import annotations

import ctypes as C

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
        ("pop_layout", C.c_int),
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


class FeDriverCfg(C.Structure):
    _fields_ = [("model", C.c_char * 32),
                ("output_dir", C.c_char * 256), ("output_name", C.c_char * 128),
                ("timeseries_file", C.c_char * 128), ("log_file", C.c_char * 128),
                ("param_file", C.c_char * 256), ("velocity_set", C.c_char * 16),
                ("domain_geometry", C.c_char * 64), ("domain_cfg_file", C.c_char * 256),
                ("fluid_initializer", C.c_char * 64), ("fluid_init_filename", C.c_char * 256),
                ("restart_file", C.c_char * 256),
                ("size_x", C.c_int), ("size_y", C.c_int), ("size_z", C.c_int),
                ("max_iterations", C.c_int64),
                ("log_skip", C.c_int), ("file_skip", C.c_int),
                ("checkpoint_skip", C.c_uint32), ("output_deflate", C.c_int), ("output_float32", C.c_int),
                ("gpu_device", C.c_int), ("logging", C.c_int), ("console", C.c_int),
                ("use_open_bnd", C.c_int), ("in_out_dir", C.c_int), ("buffer_layers", C.c_int),
                ("empty_layers", C.c_int), ("extrude_buffers", C.c_int),
                ("image_periodic", C.c_int), ("transverse_periodic", C.c_int),
                ("particles_enable", C.c_int), ("particles_number", C.c_int64),
                ("particles_init_mode", C.c_char * 32), ("particles_plane_offsets", C.c_char * 256),
                ("particles_dm_groups", C.c_char * 512),
                ("particles_int_order", C.c_int), ("particles_substeps", C.c_int), ("particles_file_skip", C.c_int),
                ("particles_dt", C.c_double),
                ("unknown_keys", C.c_int)]


BRICK = {"auto": 0, "8x8x8": 1, "16x16x1": 2, "8x8x4": 3, "16x8x8": 4}


class FeTracerConfig(C.Structure):
    _fields_ = [("substeps", C.c_int), ("order", C.c_int), ("velocity_skip", C.c_int), ("seed", C.c_uint64),
                ("stretching", C.c_int), ("phase_split", C.c_int), ("stretching_seed", C.c_uint64)]


class FeServerConfig(C.Structure):
    _fields_ = [("device", C.c_int), ("max_active", C.c_int), ("hbm_reserve_frac", C.c_double),
                ("chunk_steps", C.c_int), ("storage", C.c_int), ("fill_sites", C.c_int64),
                ("pop_layout", C.c_int), ("latency_first", C.c_int)]


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
