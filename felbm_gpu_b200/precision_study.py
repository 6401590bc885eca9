"""Error of the reduced-precision storages against FP64 (the workload's
precision study): populations stored in FP32; g as scaled FP16 / BF16
deviations from the rest state with h in FP32 (f16g, bf16g); or both as
16-bit deviations (f16s, bf16s); arithmetic in FP32 registers. Each runs
beside the FP64 engine (which matches the FP64 oracle to 1e-12) on the
same inputs.

Reported per storage: max|dc| and max|du| after the run, the relative
difference of the interface area (fluid node pairs along the axes whose c
straddles 1/2), and, for the periodic mass-corrected case, the relative
order-parameter mass drift scaled to 10^4 steps.

    python -m felbm_gpu_b200.precision_study [--size 150] [--steps 5000]

Needs a GPU; prints one JSON line per case and storage.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import sys

import numpy as np

from . import MultiPhaseGPU, OpenBoundary, _capi, default_params, geometry


def _with_storage(p, storage):
    q = _capi.FeParams()
    C.pointer(q)[0] = p
    q.storage = _capi.STORAGE[storage]
    return q


def interface_area(solid: np.ndarray, c_sites: np.ndarray) -> int:
    """Fluid node pairs along x, y, z (periodic) whose c straddles 1/2."""
    grid = np.full(solid.shape, np.nan)
    grid[solid == 0] = c_sites
    s = grid - 0.5
    n = 0
    for ax in range(3):
        if solid.shape[ax] == 1:
            continue
        t = np.roll(s, -1, axis=ax)
        n += int(np.count_nonzero((s * t) < 0))  # NaN pairs compare False
    return n


def open_case(size: int, mrt: bool, seed: int = 7):
    """The precision workload: random-field medium (corr 6, porosity 0.35,
    largest x-spanning cluster) between open inlet/outlet along x, pressure
    difference 1e-3 (in density units), contact angle 60 deg, slab start."""
    medium, por = geometry.grf((size, size, size), 6.0, 0.35, seed, flow_axis=0)
    solid = geometry.pad_open(medium, 0, 2, 2)
    inl, outl, bv, br, coord = geometry.open_lists(solid, 0, 2, split_axis=1)
    sigma, W = 1e-3, 4.0
    p = default_params(rho0=1.0, rho1=1.0, tau0=1.0, tau1=1.0, surface_tension=sigma, interface_width=W,
                       mobility_coeff=0.02, phi=6 * sigma * np.cos(np.radians(60.0)), use_mrt=int(mrt),
                       use_halfway_bb=1)
    ob = OpenBoundary(inlet=inl, outlet=outl, inlet_coord=coord, buf_verts=bv, buf_refs=br, copy_to_buffers=True,
                      use_in_prs=True, p_in=1.0 + 1e-3 / 3.0, use_out_prs=True, p_out=1.0, use_in_fluid=True,
                      use_out_fluid=True, c_out_fixed=0.0, inlet_c_a=1.0, rho_out_fixed=p.rho1)
    nx = solid.shape[2]
    c = geometry.order_parameter(solid, "slab", W, origin=(0, 0, 0), axis=0, thickness=nx // 2)
    h, g = geometry.equilibrium(c, 1.0, p.rho0, p.rho1)
    return solid, p, ob, h, g, por


def periodic_case(size: int, seed: int = 2024):
    """The production configuration (C3) at a smaller size: periodic, body
    force 1e-6, fused MRT, contact angle 45 deg, mass correction."""
    solid, por = geometry.grf((size, size, size), 6.0, 0.37, seed, flow_axis=0)
    sigma, W = 0.0083, 5.0
    p = default_params(rho0=1.0, rho1=1.0, tau0=0.9, tau1=0.9, surface_tension=sigma, interface_width=W,
                       mobility_coeff=0.02, phi=6 * sigma * np.cos(np.radians(45.0)), gx=1e-6, use_mrt=1,
                       use_halfway_bb=1, correct_op_mass=1)
    c = geometry.order_parameter(solid, "slab", W, origin=(0, 0, 0), axis=0, thickness=size // 2)
    h, g = geometry.equilibrium(c, 1.0, p.rho0, p.rho1)
    return solid, p, None, h, g, por


def run(solid, p, ob, h, g, storage, steps):
    e = MultiPhaseGPU(_with_storage(p, storage), solid)
    try:
        if ob is not None:
            e.set_open_bnd(ob)
        e.upload_state(h, g)
        if p.correct_op_mass:
            e.record_target_mass()
        m0 = e.get_target_mass() if p.correct_op_mass else None
        e.run(steps)
        f = e.download()
        m = e.current_mass() if p.correct_op_mass else None
        return f, m0, m
    finally:
        e.free()


def study(name, case, steps, storages=("f32", "f16g", "bf16g", "f16s", "bf16s")):
    solid, p, ob, h, g, por = case
    ref, m0, m_ref = run(solid, p, ob, h, g, "f64", steps)
    a_ref = interface_area(solid, ref["c"])
    out = []
    for st in ("f64",) + tuple(storages):
        f, m0s, m = (ref, m0, m_ref) if st == "f64" else run(solid, p, ob, h, g, st, steps)
        du = np.sqrt((f["ux"] - ref["ux"]) ** 2 + (f["uy"] - ref["uy"]) ** 2 + (f["uz"] - ref["uz"]) ** 2)
        area = interface_area(solid, f["c"])
        rec = {"case": name, "storage": st, "steps": steps, "sites": int(len(ref["c"])), "porosity": por,
               "max_abs_dc": float(np.max(np.abs(f["c"] - ref["c"]))), "max_abs_du": float(np.max(du)),
               "max_abs_u_fp64": float(np.max(np.sqrt(ref["ux"] ** 2 + ref["uy"] ** 2 + ref["uz"] ** 2))),
               "interface_area": area, "interface_area_rel_diff": (area - a_ref) / a_ref if a_ref else 0.0}
        if m0s is not None:
            rec["mass_drift_rel_per_1e4_steps"] = abs(m - m0s) / abs(m0s) * 1e4 / steps
        out.append(rec)
        print(json.dumps(rec), flush=True)
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=150)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--mass-steps", type=int, default=2000)
    a = ap.parse_args(argv)
    for mrt in (False, True):
        study("open %d^3 %s" % (a.size, "MRT" if mrt else "BGK"), open_case(a.size, mrt), a.steps)
    study("periodic %d^3 MRT, mass correction" % a.size, periodic_case(a.size), a.mass_steps)
    return 0


if __name__ == "__main__":
    sys.exit(main())
