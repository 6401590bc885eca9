"""Seeded parity cases shared by the tests, the golden-vector generator and
smoke(). Each case is a small lattice the CPU oracle finishes in well under a
second per step, mirroring the reference's validation matrix
(scripts/validate.sh:37-50: all-fluid and porous 'spheres' geometries, BGK and
MRT, halfway bounce-back, wetting) plus the open-boundary duct the reference
runs by hand (README.md:391-395) and the cylinder-pack / random-field media of
the measured workloads.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from felbm_gpu_b200 import OpenBoundary, default_params, geometry


@dataclass
class Case:
    name: str
    solid: np.ndarray
    params: object
    h0: np.ndarray
    g0: np.ndarray
    open_bnd: OpenBoundary | None = None
    correct_mass: bool = False
    kw: dict = field(default_factory=dict)


def _ic(solid, p, kind, width, p0=1.0, **a):
    c = geometry.order_parameter(solid, kind, width, **a)
    return geometry.equilibrium(c, p0, p.rho0, p.rho1)


def make_case(name: str, **over) -> Case:
    """Build one named case; keyword overrides go to the physics parameters."""
    if name == "fluid_bgk":          # compare_cpu_gpu geom=fluid (droplet, ratio 5, hbb off)
        solid = np.zeros((12, 12, 12), np.uint8)
        kw = dict(rho0=5.0, rho1=1.0, surface_tension=0.01, interface_width=4.0, use_halfway_bb=0)
        kw.update(over)
        p = default_params(**kw)
        h, g = _ic(solid, p, "droplet", 4.0, centre=(6, 6, 6), radius=3.0)
        return Case(name, solid, p, h, g)
    if name in ("spheres_bgk", "spheres_mrt", "spheres_mrt_wet"):  # geom=spheres (porous, halfway BB)
        solid = geometry.spheres((16, 16, 16), 3.0, 6, 3.0, 12345)
        kw = dict(rho0=5.0, rho1=1.0, surface_tension=0.01, interface_width=4.0, use_halfway_bb=1,
                  use_mrt=int(name != "spheres_bgk"))
        if name == "spheres_mrt_wet":
            kw.update(phi=6 * 0.01 * np.cos(np.pi / 3), gx=1e-5)
        kw.update(over)
        p = default_params(**kw)
        h, g = _ic(solid, p, "droplet", 4.0, centre=(8, 8, 8), radius=4.0)
        return Case(name, solid, p, h, g)
    if name == "cyl2d_mrt":           # quasi-2-D cylinder pack, slab, body force
        # rates: the production configuration's explicit s_e = s_eps = 1.19, s_q = 1.2 (nu from tau),
        # or with ref_rates=True the reference's own assignment (device_engine.cuh:625),
        # which is what the reference's kernels can run
        ref_rates = bool(over.pop("ref_rates", False))
        solid, _ = geometry.cylinders((1, 48, 64), 3.0, 6.0, 0.65, 12345)
        kw = dict(rho0=1.0, rho1=1.0, tau0=1.0, tau1=1.0, surface_tension=1e-3, interface_width=4.0,
                  mobility_coeff=0.02, use_mrt=1, use_halfway_bb=1, gx=1e-5,
                  phi=6 * 1e-3 * np.cos(np.radians(60.0)))
        kw.update(over)
        p = default_params(**kw)
        if not ref_rates:
            for k, v in ((1, 1.19), (2, 1.19), (3, 1.2)):
                p.mrt_rate_mode[k] = 2
                p.mrt_rate_value[k] = v
        h, g = _ic(solid, p, "slab", 4.0, origin=(0, 0, 0), axis=0, thickness=32)
        return Case(name, solid, p, h, g)
    if name in ("grf_mrt_mass", "grf_bgk_mass"):  # porous GRF, mass correction, wetting, body force
        solid, _ = geometry.grf((20, 20, 20), 3.0, 0.45, 7, flow_axis=0)
        kw = dict(rho0=2.0, rho1=1.0, tau0=0.8, tau1=1.0, surface_tension=5e-3, interface_width=4.0,
                  use_mrt=int(name == "grf_mrt_mass"), use_halfway_bb=1, gx=2e-5, correct_op_mass=1,
                  phi=6 * 5e-3 * np.cos(np.radians(45.0)))
        kw.update(over)
        p = default_params(**kw)
        h, g = _ic(solid, p, "slab", 4.0, origin=(0, 0, 0), axis=0, thickness=10)
        return Case(name, solid, p, h, g, correct_mass=True)
    if name == "fluid_mrt":           # all-fluid MRT: the droplet of fluid_bgk, MRT with the reference rates
        solid = np.zeros((12, 12, 12), np.uint8)
        kw = dict(rho0=5.0, rho1=1.0, surface_tension=0.01, interface_width=4.0, use_halfway_bb=0, use_mrt=1)
        kw.update(over)
        p = default_params(**kw)
        h, g = _ic(solid, p, "droplet", 4.0, centre=(6, 6, 6), radius=3.0)
        return Case(name, solid, p, h, g)
    if name == "c1_cyl2d":            # the plain-method configuration, 200 x 200 x 1
        return c1_case(**over)
    if name in ("c2_open_bgk", "c2_open_mrt"):  # the precision configuration, 150^3 open
        return c2_case(mrt=name.endswith("mrt"), **over)
    if name == "c3_grf300":           # the production configuration, 300^3 periodic
        return c3_case(**over)
    if name.startswith("openbnd"):    # compare_cpu_gpu geom=openbnd: duct, pressure inlet/outlet
        mode = int(over.pop("inlet_mode", 0))
        copybuf = bool(over.pop("copy_to_buffers", name.endswith("_buf")))
        medium = np.zeros((8, 8, 12), np.uint8)
        solid = geometry.pad_open(medium, 0, 2, 2)
        nx = solid.shape[2]
        inl, outl, bv, br, coord = geometry.open_lists(solid, 0, 2, split_axis=1)
        kw = dict(rho0=5.0, rho1=1.0, surface_tension=0.01, interface_width=4.0, use_halfway_bb=0,
                  use_mrt=int("mrt" in name))
        kw.update(over)
        p = default_params(**kw)
        ob = OpenBoundary(inlet=inl, outlet=outl, inlet_coord=coord, buf_verts=bv, buf_refs=br,
                          copy_to_buffers=copybuf, use_in_prs=True, p_in=1.003, use_out_prs=True, p_out=1.0,
                          use_in_fluid=(mode != 3), use_out_fluid=False, inlet_c_a=1.0, rho_out_fixed=p.rho0)
        if mode == 1:
            ob.inlet_mode, ob.inlet_period, ob.inlet_duty, ob.inlet_ramp = 1, 20.0, 0.5, 4.0
        elif mode == 2:
            ob.inlet_mode, ob.split_axis, ob.split_pos, ob.inlet_ramp = 2, 1, 4.0, 3.0
        elif mode == 4:
            ob.inlet_mode, ob.split_axis, ob.inlet_period, ob.inlet_duty, ob.inlet_ramp = 3, 1, 8.0, 0.5, 2.0
        h, g = _ic(solid, p, "droplet", 4.0, centre=(nx / 2, 4, 4), radius=3.0)
        return Case(name, solid, p, h, g, open_bnd=ob)
    raise KeyError(name)


CASES = ["fluid_bgk", "fluid_mrt", "spheres_bgk", "spheres_mrt", "spheres_mrt_wet", "cyl2d_mrt", "grf_mrt_mass",
         "grf_bgk_mass", "openbnd_bgk", "openbnd_mrt_buf"]

# inlet injection schedules of the open-boundary cases (the `inlet_mode`
# override): 1 alternate, 2 split, 4 stripes (reference d_inlet_gate,
# include/felbm_gpu/device_engine.cuh:699-728, modes 1, 2, 3)
INLET_MODES = {"alternate": 1, "split": 2, "stripes": 4}


def c1_case(size: int = 200, seed: int = 12345, **over) -> Case:
    """The plain-method configuration (bench.plain_workload), 200 x 200 x 1."""
    import bench
    solid, p, h, g = bench.plain_workload(size, seed, **over)
    return Case("c1_cyl2d", solid, p, h, g)


def c2_case(mrt: bool, size: int = 150, seed: int = 7, **over) -> Case:
    """The precision configuration (bench.precision_workload), 150^3 open."""
    import bench
    solid, p, ob, h, g, _ = bench.precision_workload(size, mrt, seed, **over)
    return Case("c2_open_mrt" if mrt else "c2_open_bgk", solid, p, h, g, open_bnd=ob)


def c3_case(size: int = 300, seed: int = 2024, **over) -> Case:
    """The production configuration, the benched lattice itself (bench.workload)."""
    import bench
    solid, _, p, h, g = bench.workload(size, seed, **over)
    return Case("c3_grf300", solid, p, h, g, correct_mass=True)
