"""ctypes wrapper of the reference-kernel harness (oracle/_ref/libref_kernels_*.so)
— TEST INFRASTRUCTURE ONLY.

Runs matNBI/felbm_gpu's own device_engine.cuh kernels (compiled unmodified for
sm_100a by oracle/ref/build_ref.sh) on the neighbour/case tables, streaming
table, in-place program and MRT matrices of the CPU oracle, so that the
oracle's restatement can be checked against the reference's kernels on the
same inputs. Needs a GPU.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .oracle_py import capi  # the C-ABI's layouts, without the engine library

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")


def available(precision: str = "f64") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref_kernels_{precision}.so"))


_libs: dict = {}


def _load(precision: str):
    if precision in _libs:
        return _libs[precision]
    lib = C.CDLL(os.path.join(REF_DIR, f"libref_kernels_{precision}.so"))
    vp, dp, i32p = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32)
    sig = {
        "ref_real_size": (C.c_int, []),
        "ref_create": (vp, [C.POINTER(capi.FeParams), C.c_int, C.POINTER(i32p), C.c_int, i32p, i32p,
                            C.POINTER(C.c_uint8), dp, dp]),
        "ref_set_open_bnd": (C.c_int, [vp, C.POINTER(capi.FeOpenBnd)]),
        "ref_set_forcing_factor": (None, [vp, C.c_double]),
        "ref_upload": (C.c_int, [vp, dp, dp]),
        "ref_download": (C.c_int, [vp, dp, dp]),
        "ref_step": (C.c_int, [vp]),
        "ref_record_target_mass": (None, [vp]),
        "ref_set_target_mass": (None, [vp, C.c_double]),
        "ref_apply_mass_correction": (C.c_double, [vp]),
        "ref_fields": (C.c_int, [vp, C.c_int, C.POINTER(dp)]),
        "ref_sync": (C.c_int, []),
        "ref_destroy": (None, [vp]),
    }
    for n, (r, a) in sig.items():
        getattr(lib, n).restype = r
        getattr(lib, n).argtypes = a
    _libs[precision] = lib
    return lib


_FIELDS = ("rho", "c", "ux", "uy", "uz", "p", "mu")


class RefKernels:
    """The reference's kernels in MultiPhaseGPU::step order on the oracle's tables."""

    def __init__(self, params, oracle, precision: str = "f64", inplace: bool = False):
        from .oracle_py import mrt_matrices
        self.lib = _load(precision)
        self.n = oracle.n
        self.Vn = 19 * self.n
        tabs = [np.ascontiguousarray(oracle.table(w)) for w in range(10)]
        self._keep = tabs
        arr = (C.POINTER(C.c_int32) * 10)(*[t.ctypes.data_as(C.POINTER(C.c_int32)) for t in tabs])
        M, Minv = mrt_matrices()
        M = np.ascontiguousarray(M)
        Minv = np.ascontiguousarray(Minv)
        self._keep += [M, Minv]
        prog = oracle.inplace_program() if inplace else None
        if prog is not None:
            a, b, t = prog
            self._keep += [a, b, t]
            nsops = len(a)
            pa, pb = a.ctypes.data_as(C.POINTER(C.c_int32)), b.ctypes.data_as(C.POINTER(C.c_int32))
            pt = t.ctypes.data_as(C.POINTER(C.c_uint8))
        else:
            nsops, pa, pb, pt = -1, None, None, None
        dp = C.POINTER(C.c_double)
        self._h = self.lib.ref_create(C.byref(params), self.n, arr, nsops, pa, pb, pt,
                                      M.ctypes.data_as(dp), Minv.ctypes.data_as(dp))

    def close(self):
        if getattr(self, "_h", None):
            self.lib.ref_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def set_open_bnd(self, ob):
        b, keep = ob.to_c()
        self.lib.ref_set_open_bnd(self._h, C.byref(b))
        del keep

    def set_forcing_factor(self, ff):
        self.lib.ref_set_forcing_factor(self._h, ff)

    def upload_state(self, h, g):
        h = np.ascontiguousarray(h, np.float64)
        g = np.ascontiguousarray(g, np.float64)
        dp = C.POINTER(C.c_double)
        assert self.lib.ref_upload(self._h, h.ctypes.data_as(dp), g.ctypes.data_as(dp)) == 0

    def download_state(self):
        h, g = np.empty(self.Vn), np.empty(self.Vn)
        dp = C.POINTER(C.c_double)
        assert self.lib.ref_download(self._h, h.ctypes.data_as(dp), g.ctypes.data_as(dp)) == 0
        return h, g

    def step(self, nsteps=1):
        for _ in range(nsteps):
            rc = self.lib.ref_step(self._h)
            if rc:
                raise RuntimeError(f"reference kernels: CUDA error {rc}")
        assert self.lib.ref_sync() == 0

    def record_target_mass(self):
        self.lib.ref_record_target_mass(self._h)

    def apply_mass_correction(self):
        return self.lib.ref_apply_mass_correction(self._h)

    def _fields(self, refresh):
        out = {k: np.empty(self.n) for k in _FIELDS}
        dp = C.POINTER(C.c_double)
        arr = (dp * 7)(*[out[k].ctypes.data_as(dp) for k in _FIELDS])
        assert self.lib.ref_fields(self._h, int(refresh), arr) == 0
        return out

    def fields(self):
        return self._fields(False)

    def download(self):
        return self._fields(True)
