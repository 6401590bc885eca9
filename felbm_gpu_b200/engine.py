"""Python mirror of the reference engine interface over the C-ABI.

``MultiPhaseGPU`` keeps the member names of the reference's
``struct felbm_gpu::MultiPhaseGPU`` (include/felbm_gpu/multiphase_gpu.cuh):
``init``-time construction, ``upload_state``, ``set_open_bnd``, ``step``,
``apply_mass_correction``, ``record_target_mass``, ``set_target_mass`` /
``get_target_mass``, ``current_mass``, ``download_state``, ``download``,
``flow_stats`` (+ ``_launch`` / ``_ready`` / ``_collect``), ``state_size``
and ``free``. Errors raise ``FeError`` instead of exiting the process.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _capi as capi
from ._capi import check, lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i32(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(C.POINTER(C.c_int32))


def default_params(**kw) -> capi.FeParams:
    """Reference defaults (fe_params_default) overridden by keyword cfg keys,
    then the derived kappa, beta, mobility, bnd_coeff (fe_params_derive)."""
    p = capi.FeParams()
    check(lib.fe_params_default(C.byref(p)))
    for k, v in kw.items():
        if k == "storage" and isinstance(v, str):
            v = capi.STORAGE[v]
        if k == "brick" and isinstance(v, str):
            v = capi.BRICK[v]
        if k == "pop_layout" and isinstance(v, str):
            v = {"two_buffers": 0, "in_place": 1}[v]
        if k in ("mrt_rate_mode", "mrt_rate_value"):
            arr = getattr(p, k)
            for i, x in v.items() if isinstance(v, dict) else enumerate(v):
                arr[i] = x
            continue
        if not hasattr(p, k):
            raise KeyError(f"unknown parameter {k}")
        setattr(p, k, v)
    check(lib.fe_params_derive(C.byref(p)))
    return p


def read_cfg(settings_path: str, params: capi.FeParams | None = None):
    """Read the reference driver's settings.cfg and the params.cfg it names
    (fe_cfg_read). Returns (params, open-boundary flags and values as an
    OpenBoundary without node lists, driver-level keys as a dict, the
    fast-path switch mapping as text)."""
    p = capi.FeParams()
    if params is None:
        check(lib.fe_params_default(C.byref(p)))
    else:
        C.pointer(p)[0] = params
    b = capi.FeOpenBnd()
    d = capi.FeDriverCfg()
    check(lib.fe_cfg_read(str(settings_path).encode(), C.byref(p), C.byref(b), C.byref(d)))
    drv = {}
    for k, _ in capi.FeDriverCfg._fields_:
        v = getattr(d, k)
        drv[k] = v.decode() if isinstance(v, bytes) else v
    ob = OpenBoundary(inlet=np.zeros(0, np.int32), outlet=np.zeros(0, np.int32),
                      copy_to_buffers=bool(b.copy_to_buffers), use_in_vel=bool(b.use_in_vel),
                      use_in_prs=bool(b.use_in_prs), use_in_fluid=bool(b.use_in_fluid),
                      use_out_prs=bool(b.use_out_prs), use_out_fluid=bool(b.use_out_fluid),
                      u_in=(b.u_in_x, b.u_in_y, b.u_in_z), p_in=b.p_in, p_out=b.p_out, c_out_fixed=b.c_out_fixed,
                      rho_out_fixed=b.rho_out_fixed, inlet_c_a=b.inlet_c_a, inlet_mode=b.inlet_mode,
                      split_axis=b.split_axis, inlet_period=b.inlet_period, inlet_duty=b.inlet_duty,
                      inlet_ramp=b.inlet_ramp, split_pos=b.split_pos)
    buf = C.create_string_buffer(4096)
    check(lib.fe_cfg_switch_log(C.byref(p), buf, len(buf)))
    return p, ob, drv, buf.value.decode()


def autotune(params, solid: np.ndarray, steps: int = 20, device: int = 0) -> dict:
    """Time the brick shapes and graph lengths this lattice can use and record
    the fastest for its size class (fe_autotune); engines created afterwards
    with brick = "auto" in that class take it. Returns the choice and the
    per-candidate MLUPS."""
    solid = np.ascontiguousarray(solid, np.uint8)
    nz, ny, nx = solid.shape
    r = capi.FeTuneReport()
    check(lib.fe_autotune(C.byref(params), nx, ny, nz, solid.ctypes.data_as(C.POINTER(C.c_uint8)), device, steps,
                          C.byref(r)))
    names = {v: k for k, v in capi.BRICK.items()}
    return {"brick": names[r.brick], "graph_steps": r.graph_steps,
            "candidates": [(names[r.cand_brick[i]], r.cand_graph_steps[i], r.cand_mlups[i]) for i in range(r.ncand)]}


def tune_save(path: str):
    check(lib.fe_tune_save(path.encode()))


def tune_load(path: str):
    check(lib.fe_tune_load(path.encode()))


def tune_clear():
    check(lib.fe_tune_clear())


@dataclass
class OpenBoundary:
    """Open inlet/outlet description (reference set_open_bnd + DevParams block)."""
    inlet: np.ndarray
    outlet: np.ndarray
    inlet_coord: np.ndarray | None = None
    buf_verts: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    buf_refs: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    copy_to_buffers: bool = False
    use_in_vel: bool = False
    use_in_prs: bool = False
    use_in_fluid: bool = False
    use_out_prs: bool = False
    use_out_fluid: bool = False
    u_in: tuple = (0.0, 0.0, 0.0)
    p_in: float = 0.0
    p_out: float = 0.0
    c_out_fixed: float = 0.0
    rho_out_fixed: float = 1.0
    inlet_c_a: float = 1.0
    inlet_mode: int = 0
    split_axis: int = 0
    inlet_period: float = 0.0
    inlet_duty: float = 0.5
    inlet_ramp: float = 0.0
    split_pos: float = 0.0

    def to_c(self):
        """Build the fe_open_bnd struct; returns (struct, keepalive list)."""
        keep = []
        b = capi.FeOpenBnd()
        a, pa = _i32(self.inlet); keep.append(a)
        o, po = _i32(self.outlet); keep.append(o)
        bv, pbv = _i32(self.buf_verts); keep.append(bv)
        br, pbr = _i32(self.buf_refs); keep.append(br)
        b.n_inlet, b.inlet = len(a), pa
        b.n_outlet, b.outlet = len(o), po
        b.n_buf, b.buf_verts, b.buf_refs = len(bv), pbv, pbr
        if self.inlet_coord is not None:
            ic = np.ascontiguousarray(self.inlet_coord, dtype=np.float64)
            keep.append(ic)
            b.inlet_coord = _dptr(ic)
        for k in ("copy_to_buffers", "use_in_vel", "use_in_prs", "use_in_fluid", "use_out_prs", "use_out_fluid",
                  "inlet_mode", "split_axis"):
            setattr(b, k, int(getattr(self, k)))
        b.u_in_x, b.u_in_y, b.u_in_z = self.u_in
        for k in ("p_in", "p_out", "c_out_fixed", "rho_out_fixed", "inlet_c_a", "inlet_period", "inlet_duty",
                  "inlet_ramp", "split_pos"):
            setattr(b, k, float(getattr(self, k)))
        return b, keep


class MultiPhaseGPU:
    """One lattice on one GPU (reference MultiPhaseGPU, multiphase_gpu.cuh:23)."""

    def __init__(self, params: capi.FeParams, solid: np.ndarray, device: int = -1):
        solid = np.ascontiguousarray(solid, dtype=np.uint8)
        if solid.ndim != 3:
            raise ValueError("solid must be a (nz, ny, nx) array")
        nz, ny, nx = solid.shape
        self.shape = (nz, ny, nx)
        self.params = params
        h = C.c_void_p()
        check(lib.fe_engine_create(C.byref(params), nx, ny, nz, solid.ctypes.data_as(C.POINTER(C.c_uint8)),
                                   device, C.byref(h)))
        self._h = h
        n, vn = C.c_int64(), C.c_int64()
        check(lib.fe_engine_size(self._h, C.byref(n), C.byref(vn)))
        self.n, self.Vn = n.value, vn.value

    # -- lifecycle --------------------------------------------------------
    def free(self):
        if self._h:
            # tracers on this engine use its stream: they go first
            for t in list(getattr(self, "_tracers", ())):
                t.free()
            lib.fe_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def state_size(self) -> int:
        return self.Vn

    def set_params(self, params: capi.FeParams):
        self.params = params
        check(lib.fe_set_params(self._h, C.byref(params)))

    # -- state ------------------------------------------------------------
    def upload_state(self, h: np.ndarray, g: np.ndarray):
        h = np.ascontiguousarray(h, dtype=np.float64)
        g = np.ascontiguousarray(g, dtype=np.float64)
        check(lib.fe_upload_state(self._h, _dptr(h), _dptr(g), self.Vn))

    def upload_equilibrium(self, c: np.ndarray, p=1.0):
        """The equilibrium state at rest of the per-site order parameter c
        and pressure p (an array of n values or one number), built on the
        device: the state upload_state gives for geometry.equilibrium(c, p)."""
        c = np.ascontiguousarray(c, dtype=np.float64)
        if c.size != self.n:
            raise ValueError(f"c holds {c.size} values, the lattice has {self.n} sites")
        if np.ndim(p) == 0:
            check(lib.fe_upload_equilibrium(self._h, _dptr(c), None, float(p), self.n))
        else:
            pa = np.ascontiguousarray(p, dtype=np.float64)
            if pa.size != self.n:
                raise ValueError(f"p holds {pa.size} values, the lattice has {self.n} sites")
            check(lib.fe_upload_equilibrium(self._h, _dptr(c), _dptr(pa), 0.0, self.n))

    def download_state(self, h: np.ndarray = None, g: np.ndarray = None):
        """The state as FP64 (h, g) in the reference layout f[k*n + i]. Given
        h and g (contiguous float64 arrays of 19 n entries), writes into them
        instead of new arrays: a caller that downloads repeatedly keeps its
        buffers, and the copy does not pay for touching fresh pages."""
        if h is None:
            h = np.empty(self.Vn, np.float64)
        if g is None:
            g = np.empty(self.Vn, np.float64)
        for a in (h, g):
            if a.dtype != np.float64 or a.size != self.Vn or not a.flags.c_contiguous or not a.flags.writeable:
                raise ValueError("download_state: h and g must be writable contiguous float64 arrays of 19 n")
        check(lib.fe_download_state(self._h, _dptr(h), _dptr(g), self.Vn))
        return h, g

    def set_open_bnd(self, ob: OpenBoundary):
        b, keep = ob.to_c()
        check(lib.fe_set_open_bnd(self._h, C.byref(b)))
        del keep

    # -- stepping ---------------------------------------------------------
    def step(self, nsteps: int = 1):
        check(lib.fe_step(self._h, nsteps))

    def run(self, nsteps: int):
        check(lib.fe_run(self._h, nsteps))

    def set_forcing_factor(self, ff: float):
        check(lib.fe_set_forcing_factor(self._h, ff))

    def set_time(self, t: int):
        check(lib.fe_set_time(self._h, t))

    def get_time(self) -> int:
        t = C.c_int64()
        check(lib.fe_get_time(self._h, C.byref(t)))
        return t.value

    def apply_mass_correction(self, want_drift: bool = True):
        d = C.c_double()
        check(lib.fe_apply_mass_correction(self._h, C.byref(d) if want_drift else None))
        return d.value if want_drift else None

    def record_target_mass(self):
        check(lib.fe_record_target_mass(self._h))

    def set_target_mass(self, m0: float):
        check(lib.fe_set_target_mass(self._h, m0))

    def get_target_mass(self) -> float:
        d = C.c_double()
        check(lib.fe_get_target_mass(self._h, C.byref(d)))
        return d.value

    def current_mass(self) -> float:
        d = C.c_double()
        check(lib.fe_current_mass(self._h, C.byref(d)))
        return d.value

    # -- readout ----------------------------------------------------------
    def download(self) -> dict:
        """Fields c, rho, ux, uy, uz, p, mu refreshed from the current state."""
        out = {k: np.empty(self.n, np.float64) for k in ("rho", "c", "ux", "uy", "uz", "p", "mu")}
        f = capi.FeFields(*[_dptr(out[k]) for k in ("rho", "c", "ux", "uy", "uz", "p", "mu")])
        check(lib.fe_download_fields(self._h, C.byref(f)))
        return out

    def layout(self):
        """(brick name, steps per graph launch) this engine runs with."""
        b, g = C.c_int32(), C.c_int32()
        check(lib.fe_engine_layout(self._h, C.byref(b), C.byref(g)))
        return {v: k for k, v in capi.BRICK.items()}[b.value], g.value

    def flow_stats(self) -> np.ndarray:
        out = np.empty(6, np.float64)
        check(lib.fe_flow_stats(self._h, _dptr(out)))
        return out

    def flow_stats_launch(self):
        check(lib.fe_flow_stats_launch(self._h))

    def flow_stats_ready(self) -> bool:
        r = C.c_int()
        check(lib.fe_flow_stats_ready(self._h, C.byref(r)))
        return bool(r.value)

    def flow_stats_collect(self) -> np.ndarray:
        out = np.empty(6, np.float64)
        check(lib.fe_flow_stats_collect(self._h, _dptr(out)))
        return out

    # -- diagnostics ------------------------------------------------------
    def time_run(self, nsteps: int) -> float:
        ms = C.c_float()
        check(lib.fe_time_run(self._h, nsteps, C.byref(ms)))
        return ms.value

    def time_kernels(self, nsteps: int) -> np.ndarray:
        ms = (C.c_float * 5)()
        check(lib.fe_time_kernels(self._h, nsteps, ms, 5))
        return np.array(ms[:], dtype=np.float64)

    def launch_count(self) -> int:
        c = C.c_int64()
        check(lib.fe_launch_count(self._h, C.byref(c)))
        return c.value


class Batch:
    """Many engines advanced together (fe_batch_*): one launch per pass over
    all members, CUDA graphs; each member gets the result it gets alone."""

    def __init__(self, device: int = -1):
        h = C.c_void_p()
        check(lib.fe_batch_create(device, C.byref(h)))
        self._h = h
        self.members: list[MultiPhaseGPU] = []

    def add(self, eng: MultiPhaseGPU):
        check(lib.fe_batch_add(self._h, eng._h))
        self.members.append(eng)

    def remove(self, eng: MultiPhaseGPU):
        check(lib.fe_batch_remove(self._h, eng._h))
        self.members.remove(eng)

    def size(self) -> tuple[int, int]:
        m, n = C.c_int(), C.c_int64()
        check(lib.fe_batch_size(self._h, C.byref(m), C.byref(n)))
        return m.value, n.value

    def run(self, nsteps: int):
        check(lib.fe_batch_run(self._h, nsteps))

    def time_run(self, nsteps: int) -> float:
        ms = C.c_float()
        check(lib.fe_batch_time_run(self._h, nsteps, C.byref(ms)))
        return ms.value

    def launch_count(self) -> int:
        c = C.c_int64()
        check(lib.fe_batch_launch_count(self._h, C.byref(c)))
        return c.value

    def free(self):
        if self._h:
            lib.fe_batch_destroy(self._h)
            self._h = None
            self.members = []

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
