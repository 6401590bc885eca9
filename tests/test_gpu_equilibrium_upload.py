"""The equilibrium state at rest built on the device (fe_upload_equilibrium)
against the host-built state uploaded through fe_upload_state: the stored
state, its download and the state after a few steps bit-equal, for every
storage, both population layouts, a uniform and a per-site pressure, and
lattices below and above the size where the FP32-arithmetic storages move
FP32 values across the link."""
import ctypes as C

import numpy as np
import pytest

from felbm_gpu_b200 import MultiPhaseGPU, default_params, geometry
from felbm_gpu_b200 import _capi as capi
from felbm_gpu_b200._capi import FeError

pytestmark = pytest.mark.gpu


def _lattice(big: bool):
    if big:  # 64^3 porous: 19 n FP32 values above 4 MB
        return geometry.grf((64, 64, 64), 4.0, 0.45, 5, flow_axis=0)[0]
    return geometry.spheres((16, 16, 16), 3.0, 6, 3.0, 12345)


def _states(solid, p, c, pres, layout):
    """(host-built upload, device-built upload): download right after the
    upload and after 5 steps (the second with a queued mass correction)."""
    out = []
    for device in (False, True):
        q = capi.FeParams()
        C.pointer(q)[0] = p
        q.pop_layout = layout
        e = MultiPhaseGPU(q, solid)
        try:
            if device:
                e.upload_equilibrium(c, pres)
            else:
                e.upload_state(*geometry.equilibrium(c, pres, q.rho0, q.rho1))
            first = np.concatenate(e.download_state())
            e.record_target_mass()
            e.run(5)
            e.apply_mass_correction(want_drift=False)
            out.append((first, np.concatenate(e.download_state()), e.current_mass()))
        finally:
            e.free()
    return out


@pytest.mark.parametrize("storage", ["f64", "f32", "f16g", "bf16g", "f16s", "bf16s"])
@pytest.mark.parametrize("big", [False, True])
def test_device_equilibrium_equals_host_state(require_gpu, storage, big):
    solid = _lattice(big)
    p = default_params(rho0=2.0, rho1=1.0, use_mrt=1, use_halfway_bb=1, correct_op_mass=1,
                       surface_tension=5e-3, interface_width=4.0, gx=1e-5, storage=storage)
    e = MultiPhaseGPU(p, solid)
    n = e.n
    e.free()
    rng = np.random.default_rng(7)
    c = 0.5 + 0.5 * np.tanh(2.0 * rng.standard_normal(n))
    host, dev = _states(solid, p, c, 1.0, 0)
    for a, b in zip(host[:2], dev[:2]):
        assert np.array_equal(a, b)
    assert host[2] == dev[2]


@pytest.mark.parametrize("storage", ["f64", "f32"])
def test_device_equilibrium_per_site_pressure_and_in_place(require_gpu, storage):
    solid = _lattice(True)
    p = default_params(rho0=1.0, rho1=1.0, use_mrt=1, use_halfway_bb=1, correct_op_mass=1,
                       surface_tension=5e-3, interface_width=4.0, gx=1e-5, storage=storage)
    e = MultiPhaseGPU(p, solid)
    n = e.n
    e.free()
    rng = np.random.default_rng(8)
    c = geometry.order_parameter(solid, "slab", 4.0, origin=(0.0, 0.0, 0.0), axis=0, thickness=20.0)
    pres = 1.0 + 0.01 * rng.standard_normal(n)
    for layout in (0, 1):
        host, dev = _states(solid, p, c, pres, layout)
        for a, b in zip(host[:2], dev[:2]):
            assert np.array_equal(a, b), layout
        assert host[2] == dev[2]


def test_device_equilibrium_size_checks(require_gpu):
    solid = _lattice(False)
    e = MultiPhaseGPU(default_params(storage="f32"), solid)
    try:
        with pytest.raises(ValueError):
            e.upload_equilibrium(np.zeros(e.n + 1))
        with pytest.raises(ValueError):
            e.upload_equilibrium(np.zeros(e.n), np.ones(e.n - 1))
        c = np.zeros(e.n)
        assert capi.lib.fe_upload_equilibrium(e._h, c.ctypes.data_as(C.POINTER(C.c_double)), None, 1.0,
                                              e.n + 1) != 0
        with pytest.raises(FeError):
            capi.check(capi.lib.fe_upload_equilibrium(e._h, None, None, 1.0, e.n))
    finally:
        e.free()
