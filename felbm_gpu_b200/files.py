"""The reference driver's files (fields, geometry, checkpoint, particles) from
Python, written and read by the library's own HDF5 module."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._capi import check, lib

_dp = C.POINTER(C.c_double)
_i32 = C.POINTER(C.c_int32)
_i64 = C.POINTER(C.c_int64)
_DT = {0: np.float64, 1: np.float32, 2: np.int32, 3: np.uint32}


def write_fields(engine, path: str, float32: bool = False, deflate: int = 0):
    """Field file <output_name>_<iter>.h5: output_float32 and output_deflate
    (gzip level 0-9, one chunk per dataset) as the reference's cfg keys."""
    check(lib.fe_write_fields_h5(engine._h, path.encode(), int(float32), int(deflate)))


def write_dataset(path: str, name: str, arr: np.ndarray, deflate: int = 0):
    """A new file holding one 1-D or 2-D array (float64, float32, int32 or
    uint32), contiguous or (deflate 1-9) one gzip-filtered chunk."""
    arr = np.ascontiguousarray(arr)
    code = {np.dtype(np.float64): 0, np.dtype(np.float32): 1, np.dtype(np.int32): 2, np.dtype(np.uint32): 3}
    if arr.dtype not in code or arr.ndim not in (1, 2):
        raise ValueError("write_dataset: 1-D or 2-D float64, float32, int32 or uint32")
    dims = np.array(arr.shape, np.int64)
    check(lib.fe_h5_write_dataset(path.encode(), name.encode(), code[arr.dtype], arr.ndim,
                                  dims.ctypes.data_as(_i64), arr.ctypes.data_as(C.c_void_p), int(deflate)))


def write_geometry(path: str, solid: np.ndarray):
    solid = np.ascontiguousarray(solid, np.uint8)
    nz, ny, nx = solid.shape
    check(lib.fe_write_geometry_h5(path.encode(), solid.ctypes.data_as(C.POINTER(C.c_uint8)), nx, ny, nz))


def write_checkpoint(engine, path: str, step: int):
    check(lib.fe_checkpoint_write(engine._h, path.encode(), step))


def read_checkpoint(engine, path: str) -> int:
    st = C.c_uint32()
    check(lib.fe_checkpoint_read(engine._h, path.encode(), C.byref(st)))
    return st.value


def write_particles(path: str, pos, vel=None, ids=None, dm=None, plane_id=None, rho_hat=None, log_rho=None):
    pos = np.ascontiguousarray(pos, np.float64).reshape(3, -1)
    n = pos.shape[1]
    keep = [pos]

    def ptr(a, dt, t):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dt)
        keep.append(a)
        return a.ctypes.data_as(t)
    check(lib.fe_write_particles_h5(path.encode(), n, pos.ctypes.data_as(_dp), ptr(vel, np.float64, _dp),
                                    ptr(ids, np.int64, _i64), ptr(dm, np.float64, _dp),
                                    ptr(plane_id, np.int32, _i32), ptr(rho_hat, np.float64, _dp),
                                    ptr(log_rho, np.float64, _dp)))


def write_series(path: str, iteration: int, stats, n_sites: int, header: bool = False):
    """One line of series.txt from the six flow-statistics sums (header:
    truncate and write the column line first)."""
    st = np.ascontiguousarray(stats, np.float64)
    check(lib.fe_write_series(path.encode(), int(header), int(iteration), st.ctypes.data_as(_dp), int(n_sites)))


def write_stretching(path: str, rows, header: bool = False):
    """Rows (k, 9) of Tracers.stretch_rows() appended to stretching.txt."""
    r = np.ascontiguousarray(rows, np.float64).reshape(-1, 9)
    check(lib.fe_write_stretching(path.encode(), int(header), r.ctypes.data_as(_dp), len(r)))


def read_dataset(path: str, name: str) -> np.ndarray:
    t, rank = C.c_int(), C.c_int()
    dims = (C.c_int64 * 2)()
    check(lib.fe_h5_read_dataset(path.encode(), name.encode(), C.byref(t), dims, C.byref(rank), None, 0))
    shape = tuple(dims[a] for a in range(rank.value))
    out = np.empty(shape, _DT[t.value])
    check(lib.fe_h5_read_dataset(path.encode(), name.encode(), C.byref(t), dims, C.byref(rank),
                                 out.ctypes.data_as(C.c_void_p), out.nbytes))
    return out
