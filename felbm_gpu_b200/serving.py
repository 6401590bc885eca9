"""Serving: the native request loop (fe_server_*) from Python.

Solves are submitted at any time; the loop admits them while a slot and
device memory are free, advances every admitted solve together (one batch,
continuous batching between chunks of steps) and retires each on its step
count or convergence test. Each result is the one the solve gets alone.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _capi as capi
from ._capi import check, lib

_u8 = C.POINTER(C.c_uint8)
_dp = C.POINTER(C.c_double)


@dataclass
class Result:
    id: int
    status: int
    message: str
    sites: int
    steps_done: int
    t_submit: float
    t_admit: float
    t_done: float
    mass0: float
    mass_final: float
    stats: np.ndarray
    fields: dict = field(default_factory=dict)

    @property
    def time_to_result(self) -> float:
        return self.t_done - self.t_submit


class Server:
    """Native request loop on device `device` (fe_server_create)."""

    def __init__(self, storage: str = "f32", device: int = 0, max_active: int = 0,
                 hbm_reserve_frac: float = 0.1, chunk_steps: int = 100, fill_sites: int = 2_000_000,
                 pop_layout: str = "two_buffers", latency_first: bool = False):
        cfg = capi.FeServerConfig(device, max_active, hbm_reserve_frac, chunk_steps, capi.STORAGE[storage],
                                  fill_sites, {"two_buffers": 0, "in_place": 1}[pop_layout], int(latency_first))
        h = C.c_void_p()
        check(lib.fe_server_create(C.byref(cfg), C.byref(h)))
        self._h = h

    def submit(self, rid: int, params: capi.FeParams, solid: np.ndarray, steps: int, *, h0=None, g0=None,
               init: tuple | None = None, init_width: float = 4.0, init_p: float = 1.0, conv_tol: float = 0.0,
               want_fields: bool = True):
        """Queue one solve. The initial state is (h0, g0) in the reference
        layout, or built on the server from init = (kind, a[0..4])
        (fe_init_order_parameter) and the pressure level init_p."""
        solid = np.ascontiguousarray(solid, np.uint8)
        nz, ny, nx = solid.shape
        r = capi.FeRequest()
        r.id = rid
        r.params = params
        r.nx, r.ny, r.nz = nx, ny, nz
        r.solid = solid.ctypes.data_as(_u8)
        keep = [solid]
        if h0 is not None:
            h0 = np.ascontiguousarray(h0, np.float64)
            g0 = np.ascontiguousarray(g0, np.float64)
            keep += [h0, g0]
            r.h0, r.g0 = h0.ctypes.data_as(_dp), g0.ctypes.data_as(_dp)
        else:
            kind, a = init if init is not None else (0, (0.0,))
            r.init_kind = kind
            for i, v in enumerate(a):
                r.init_a[i] = v
        r.init_width = init_width
        r.init_p = init_p
        r.steps = steps
        r.conv_tol = conv_tol
        r.want_fields = 1 if want_fields else 0
        check(lib.fe_server_submit(self._h, C.byref(r)))  # copies the arrays
        del keep

    def poll(self, max_results: int = 64) -> list[Result]:
        buf = (capi.FeResult * max_results)()
        n = C.c_int()
        check(lib.fe_server_poll(self._h, buf, max_results, C.byref(n)))
        out = []
        for q in range(n.value):
            r = buf[q]
            fields = {}
            if r.c:
                for k in ("rho", "c", "ux", "uy", "uz", "p"):
                    ptr = getattr(r, k)
                    fields[k] = np.ctypeslib.as_array(ptr, shape=(r.sites,)).copy()
            out.append(Result(r.id, r.status, r.message.decode(errors="replace"), r.sites, r.steps_done,
                              r.t_submit, r.t_admit, r.t_done, r.mass0, r.mass_final,
                              np.array(r.stats[:]), fields))
            lib.fe_server_free_result(C.byref(r))
        return out

    def wait_idle(self, timeout: float = 600.0):
        check(lib.fe_server_wait_idle(self._h, timeout))

    def stats(self) -> dict:
        st = capi.FeServerStats()
        check(lib.fe_server_get_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in capi.FeServerStats._fields_}

    def close(self):
        if self._h:
            lib.fe_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
