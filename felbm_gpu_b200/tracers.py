"""GPU tracers (fe_tracers_*) from Python: seeding, diffusivity ladders and
the per-step advance beside an engine (reference particle tracking,
README "Particle tracking"; driver felbm_gpu_main.cu:421-581,752-777)."""
from __future__ import annotations

import ctypes as C
import weakref

import numpy as np

from . import _capi as capi
from ._capi import check, lib

_dp = C.POINTER(C.c_double)
_u8 = C.POINTER(C.c_uint8)
_i32 = C.POINTER(C.c_int32)
_i64 = C.POINTER(C.c_int64)


def seed(solid: np.ndarray, count: int, mode: str = "volume", axis: int = 0, offsets=(), rng_seed: int = 0):
    """Seed positions (3, N) and plane ids (N,): mode 'volume' (count tracers
    in the fluid) or 'plane' (count per plane normal to `axis` at each offset)."""
    solid = np.ascontiguousarray(solid, np.uint8)
    nz, ny, nx = solid.shape
    m = 0 if mode == "volume" else 1
    offs = np.ascontiguousarray(np.asarray(offsets if m else [0.0], np.float64))
    planes = len(offs) if m else 1
    total = count * planes
    pos = np.empty(3 * total, np.float64)
    pid = np.empty(total, np.int32)
    check(lib.fe_tracers_seed(solid.ctypes.data_as(_u8), nx, ny, nz, m, axis, offs.ctypes.data_as(_dp), planes, count,
                              rng_seed, pos.ctypes.data_as(_dp), pid.ctypes.data_as(_i32)))
    return pos.reshape(3, total), pid


def dm_ladder(groups, plane_id: np.ndarray) -> np.ndarray:
    """Per-tracer diffusivity from groups [(Dm, count), ...] (reference
    particles_dm_groups). When the counts sum to the tracers of one plane the
    ladder is applied within each plane (crossed design), else across all."""
    plane_id = np.asarray(plane_id)
    ladder = np.concatenate([np.full(int(c), float(d)) for d, c in groups]) if groups else np.zeros(0)
    n = len(plane_id)
    planes = np.unique(plane_id)
    per = n // max(len(planes), 1)
    out = np.zeros(n)
    if len(ladder) == per and per * len(planes) == n:
        for p in planes:
            idx = np.nonzero(plane_id == p)[0]
            out[idx] = ladder
    else:
        k = min(len(ladder), n)
        out[:k] = ladder[:k]
    return out


STRETCH_COLUMNS = ("step", "lambda", "mean_log_rho", "var_log_rho", "n_active", "lambda_w", "lambda_nw", "n_w",
                   "n_nw")


class Tracers:
    """Tracers of one engine; call step() after each engine step. With
    stretching=True every tracer carries a material line element and each
    step leaves a row of the stretching time series (STRETCH_COLUMNS),
    drained by stretch_rows(); phase_split=True splits lambda by phase."""

    def __init__(self, engine, pos: np.ndarray, dm, ids=None, substeps: int = 1, order: int = 2,
                 velocity_skip: int = 1, rng_seed: int = 0, stretching: bool = False, phase_split: bool = True,
                 stretching_seed: int = 20260801):
        pos = np.ascontiguousarray(pos, np.float64).reshape(3, -1)
        self.n = pos.shape[1]
        dm = np.ascontiguousarray(np.broadcast_to(np.asarray(dm, np.float64), (self.n,)))
        cfg = capi.FeTracerConfig(substeps, order, velocity_skip, rng_seed, int(stretching),
                                  int(stretching and phase_split), stretching_seed)
        idp = None
        if ids is not None:
            ids = np.ascontiguousarray(ids, np.int64)
            idp = ids.ctypes.data_as(_i64)
        h = C.c_void_p()
        check(lib.fe_tracers_create(engine._h, C.byref(cfg), self.n, pos.ctypes.data_as(_dp), dm.ctypes.data_as(_dp),
                                    idp, C.byref(h)))
        self._h = h
        self.engine = engine  # kept alive: tracers use the engine's stream
        if not hasattr(engine, "_tracers"):
            engine._tracers = weakref.WeakSet()
        engine._tracers.add(self)

    def step(self):
        check(lib.fe_tracers_step(self._h))

    def download(self):
        pos = np.empty(3 * self.n, np.float64)
        vel = np.empty(3 * self.n, np.float64)
        check(lib.fe_tracers_download(self._h, pos.ctypes.data_as(_dp), vel.ctypes.data_as(_dp)))
        return pos.reshape(3, self.n), vel.reshape(3, self.n)

    def stretch_rows(self, max_rows: int = 1 << 20) -> np.ndarray:
        """Rows (k, 9) made since the last call, oldest first."""
        out = np.empty((max(int(max_rows), 1), 9), np.float64)
        cnt = C.c_int64()
        check(lib.fe_tracers_stretch_rows(self._h, out.ctypes.data_as(_dp), int(max_rows), C.byref(cnt)))
        return out[:cnt.value].copy()

    def stretch_state(self):
        """(rho_hat (3, n), log_rho (n,))."""
        rh = np.empty(3 * self.n, np.float64)
        lr = np.empty(self.n, np.float64)
        check(lib.fe_tracers_stretch_state(self._h, rh.ctypes.data_as(_dp), lr.ctypes.data_as(_dp)))
        return rh.reshape(3, self.n), lr

    def set_stretch_state(self, rho_hat, log_rho):
        rh = np.ascontiguousarray(rho_hat, np.float64).reshape(-1)
        lr = np.ascontiguousarray(log_rho, np.float64).reshape(-1)
        check(lib.fe_tracers_set_stretch_state(self._h, rh.ctypes.data_as(_dp), lr.ctypes.data_as(_dp)))

    def set_velocity(self, u=None, c=None):
        """Advect on node-indexed u (3, nodes) (and order parameter c (nodes,))
        from now on; None returns to the engine's velocity."""
        if u is None:
            check(lib.fe_tracers_set_velocity(self._h, None, None))
            return
        u = np.ascontiguousarray(u, np.float64).reshape(-1)
        cp = None
        if c is not None:
            c = np.ascontiguousarray(c, np.float64).reshape(-1)
            cp = c.ctypes.data_as(_dp)
        check(lib.fe_tracers_set_velocity(self._h, u.ctypes.data_as(_dp), cp))

    def free(self):
        if getattr(self, "_h", None):
            lib.fe_tracers_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
