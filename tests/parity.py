"""Runners that advance the same case through the B200 engine, the CPU oracle
and the reference's own kernels, for the parity tests."""
from __future__ import annotations

import ctypes as C

import numpy as np

from cases import Case
from felbm_gpu_b200 import MultiPhaseGPU, _capi
from oracle.oracle_py import Oracle


def with_storage(params, storage: str):
    p = _capi.FeParams()
    C.pointer(p)[0] = params
    p.storage = _capi.STORAGE[storage]
    return p


def run_engine(case: Case, steps: int, storage: str = "f64", mode: str = "run"):
    """Upload the case, run `steps` steps (fe_run, or fe_step + correction
    calls when mode='step'), return post-step state and refreshed fields."""
    e = MultiPhaseGPU(with_storage(case.params, storage), case.solid)
    try:
        if case.open_bnd is not None:
            e.set_open_bnd(case.open_bnd)
        e.upload_state(case.h0, case.g0)
        if case.correct_mass:
            e.record_target_mass()
        if mode == "run":
            e.run(steps)
        else:
            for _ in range(steps):
                e.step(1)
                e.apply_mass_correction(want_drift=False)
        h, g = e.download_state()
        stats = e.flow_stats()
        f = e.download()
        return h, g, f, stats, e.launch_count()
    finally:
        e.free()


def run_oracle(case: Case, steps: int, inplace: bool = False):
    o = Oracle(case.params, case.solid, inplace=inplace)
    if case.open_bnd is not None:
        o.set_open_bnd(case.open_bnd)
    o.upload_state(case.h0, case.g0)
    if case.correct_mass:
        o.record_target_mass()
    o.run(steps, 0)
    h, g = o.download_state()
    stats = o.flow_stats()
    f = o.download()
    return h, g, f, stats


def maxdiff(a, b) -> float:
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) if len(a) else 0.0


def reldiff(a, b) -> float:
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return maxdiff(a, b) / scale
