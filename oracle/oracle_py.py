"""ctypes wrapper of the CPU oracle (liboracle.so) — TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg to
compare against; the product never imports it. The struct layouts are the C-ABI's
(include/felbm_b200.h), taken from felbm_gpu_b200/_abi.py, which loads no
library: a process that only runs the oracle never loads the engine.
"""
from __future__ import annotations

import ctypes as C
import importlib.util
import os
import subprocess
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))


def _abi():
    """felbm_gpu_b200._abi without importing the package (whose import loads
    the engine library); registered under its package name, so a later
    import of the package shares the same structure types."""
    name = "felbm_gpu_b200._abi"
    if name not in sys.modules:
        path = os.path.join(os.path.dirname(_HERE), "felbm_gpu_b200", "_abi.py")
        spec = importlib.util.spec_from_file_location(name, path)
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


capi = _abi()

LIB_PATH = os.path.join(_HERE, "liboracle.so")


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


if not os.path.exists(LIB_PATH):
    build()
_lib = C.CDLL(LIB_PATH)
_vp, _dp, _i64p = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64)
_sig = {
    "or_create": (_vp, [C.POINTER(capi.FeParams), C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint8), C.c_int]),
    "or_destroy": (None, [_vp]),
    "or_n": (C.c_int64, [_vp]),
    "or_site_nodes": (None, [_vp, _i64p]),
    "or_set_open_bnd": (C.c_int, [_vp, C.POINTER(capi.FeOpenBnd)]),
    "or_set_params": (None, [_vp, C.POINTER(capi.FeParams)]),
    "or_upload": (None, [_vp, _dp, _dp]),
    "or_download": (None, [_vp, _dp, _dp]),
    "or_set_forcing_factor": (None, [_vp, C.c_double]),
    "or_step": (None, [_vp]),
    "or_apply_mass_correction": (C.c_double, [_vp]),
    "or_record_target_mass": (None, [_vp]),
    "or_target_mass": (C.c_double, [_vp]),
    "or_set_target_mass": (None, [_vp, C.c_double]),
    "or_current_mass": (C.c_double, [_vp]),
    "or_fields": (None, [_vp, C.POINTER(capi.FeFields)]),
    "or_download_fields": (None, [_vp, C.POINTER(capi.FeFields)]),
    "or_flow_stats": (None, [_vp, _dp]),
    "or_inplace_counts": (None, [_vp, _i64p]),
    "or_table": (None, [_vp, C.c_int, C.POINTER(C.c_int32)]),
    "or_run": (None, [_vp, C.c_int, C.c_int64]),
    "or_mrt_matrices": (None, [_dp, _dp]),
    "or_threads": (C.c_int, []),
    "or_set_threads": (None, [C.c_int]),
    "or_inplace_program": (C.c_int64, [_vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_uint8)]),
}
for _n, (_r, _a) in _sig.items():
    getattr(_lib, _n).restype = _r
    getattr(_lib, _n).argtypes = _a

_FIELDS = ("rho", "c", "ux", "uy", "uz", "p", "mu")


def _d(a):
    return a.ctypes.data_as(_dp)


class Oracle:
    """FP64 CPU restatement of the reference step on the reference's tables."""

    def __init__(self, params, solid: np.ndarray, inplace: bool = False):
        solid = np.ascontiguousarray(solid, np.uint8)
        nz, ny, nx = solid.shape
        self._h = _lib.or_create(C.byref(params), nx, ny, nz, solid.ctypes.data_as(C.POINTER(C.c_uint8)),
                                 int(inplace))
        self.n = _lib.or_n(self._h)
        self.Vn = 19 * self.n

    def __del__(self):
        if getattr(self, "_h", None):
            _lib.or_destroy(self._h)
            self._h = None

    def set_params(self, params):
        _lib.or_set_params(self._h, C.byref(params))

    def set_open_bnd(self, ob):
        b, keep = ob.to_c()
        _lib.or_set_open_bnd(self._h, C.byref(b))
        del keep

    def upload_state(self, h, g):
        h = np.ascontiguousarray(h, np.float64)
        g = np.ascontiguousarray(g, np.float64)
        _lib.or_upload(self._h, _d(h), _d(g))

    def download_state(self):
        h, g = np.empty(self.Vn), np.empty(self.Vn)
        _lib.or_download(self._h, _d(h), _d(g))
        return h, g

    def set_forcing_factor(self, ff):
        _lib.or_set_forcing_factor(self._h, ff)

    def step(self, nsteps=1):
        for _ in range(nsteps):
            _lib.or_step(self._h)

    def run(self, nsteps, t0=0):
        _lib.or_run(self._h, nsteps, t0)

    def apply_mass_correction(self):
        return _lib.or_apply_mass_correction(self._h)

    def record_target_mass(self):
        _lib.or_record_target_mass(self._h)

    def get_target_mass(self):
        return _lib.or_target_mass(self._h)

    def set_target_mass(self, m0):
        _lib.or_set_target_mass(self._h, m0)

    def current_mass(self):
        return _lib.or_current_mass(self._h)

    def _grab(self, fn):
        out = {k: np.empty(self.n) for k in _FIELDS}
        f = capi.FeFields(*[_d(out[k]) for k in _FIELDS])
        fn(self._h, C.byref(f))
        return out

    def fields(self):
        return self._grab(_lib.or_fields)

    def download(self):
        return self._grab(_lib.or_download_fields)

    def flow_stats(self):
        out = np.empty(6)
        _lib.or_flow_stats(self._h, _d(out))
        return out

    def inplace_counts(self):
        out = np.empty(3, np.int64)
        _lib.or_inplace_counts(self._h, out.ctypes.data_as(_i64p))
        return out

    def table(self, which: int) -> np.ndarray:
        size = (19 if which >= 8 else 18) * self.n
        out = np.empty(size, np.int32)
        _lib.or_table(self._h, which, out.ctypes.data_as(C.POINTER(C.c_int32)))
        return out

    def inplace_program(self):
        m = _lib.or_inplace_program(self._h, None, None, None)
        if m < 0:
            return None
        a, b, t = np.empty(m, np.int32), np.empty(m, np.int32), np.empty(m, np.uint8)
        _lib.or_inplace_program(self._h, a.ctypes.data_as(C.POINTER(C.c_int32)),
                                b.ctypes.data_as(C.POINTER(C.c_int32)), t.ctypes.data_as(C.POINTER(C.c_uint8)))
        return a, b, t

    def site_nodes(self):
        out = np.empty(self.n, np.int64)
        _lib.or_site_nodes(self._h, out.ctypes.data_as(_i64p))
        return out


def threads() -> int:
    return _lib.or_threads()


def set_threads(n: int):
    _lib.or_set_threads(int(n))


def mrt_matrices():
    M, Minv = np.empty(361), np.empty(361)
    _lib.or_mrt_matrices(_d(M), _d(Minv))
    return M.reshape(19, 19), Minv.reshape(19, 19)
