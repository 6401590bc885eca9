"""Serving (fe_server_*): the native request loop. Each served result must be
bit-for-bit the result of the same solve run alone through the plain engine
(continuous batching changes when a solve runs, not what it computes);
admission must respect the slot limit and the device-memory reserve; solves
submitted while others run must join them."""
import time

import numpy as np
import pytest

from felbm_gpu_b200 import MultiPhaseGPU, default_params, geometry
from felbm_gpu_b200.serving import Server
from parity import with_storage

pytestmark = pytest.mark.gpu


def solve_spec(k: int):
    """A small solve of the sweep kind: 2-D cylinder pack or 3-D random
    field, contact angle and mobility drawn from k."""
    rng = np.random.default_rng(1000 + k)
    theta = rng.uniform(30, 150)
    mob = rng.uniform(0.005, 0.05)
    sigma, W = 1e-3, 4.0
    if k % 2 == 0:
        L = int(rng.choice([48, 64, 80]))
        solid, _ = geometry.cylinders((1, L, L), 3.0, 6.0, 0.6, seed=k)
    else:
        L = int(rng.choice([24, 32]))
        solid, _ = geometry.grf((L, L, L), 4.0, 0.5, seed=k, flow_axis=0)
    init = (1, (0.0, 0.0, 0.0, 0.0, L / 2))
    p = default_params(rho0=1.0, rho1=1.0, tau0=1.0, tau1=1.0, surface_tension=sigma, interface_width=W,
                       mobility_coeff=mob, phi=6 * sigma * np.cos(np.radians(theta)), gx=1e-6, use_mrt=1,
                       correct_op_mass=1)
    steps = int(rng.integers(20, 60))
    return p, solid, init, W, steps


def alone(p, solid, init, W, steps, storage):
    kind, a = init
    c = geometry.order_parameter(solid, "slab", W, origin=a[:3], axis=int(a[3]), thickness=a[4])
    h0, g0 = geometry.equilibrium(c, 1.0, p.rho0, p.rho1)
    e = MultiPhaseGPU(with_storage(p, storage), solid)
    try:
        e.upload_state(h0, g0)
        e.record_target_mass()
        e.run(steps)
        return e.download(), e.current_mass()
    finally:
        e.free()


def collect(srv, count, timeout=300.0):
    out, t0 = [], time.time()
    while len(out) < count and time.time() - t0 < timeout:
        out += srv.poll()
        time.sleep(0.01)
    return out


@pytest.mark.parametrize("storage,latency_first", [("f32", False), ("f64", False), ("f32", True)])
def test_served_equals_alone(require_gpu, storage, latency_first):
    """Each served result bit-equal to the solve alone, with the default
    chunks and with latency-first chunks (which split the resident solves
    into smaller batches)."""
    specs = [solve_spec(k) for k in range(8)]
    srv = Server(storage=storage, max_active=3, chunk_steps=16, latency_first=latency_first)
    try:
        for k in range(4):
            p, solid, init, W, steps = specs[k]
            srv.submit(k, p, solid, steps, init=init, init_width=W)
        time.sleep(0.05)            # the rest arrive while the first ones run
        for k in range(4, 8):
            p, solid, init, W, steps = specs[k]
            srv.submit(k, p, solid, steps, init=init, init_width=W)
        res = collect(srv, 8)
        st = srv.stats()
    finally:
        srv.close()
    assert len(res) == 8
    assert st["peak_active"] <= 3 and st["completed"] == 8
    for r in res:
        assert r.status == 0, r.message
        p, solid, init, W, steps = specs[r.id]
        assert r.steps_done == steps
        f, m_alone = alone(p, solid, init, W, steps, storage)
        for k in ("c", "rho", "ux", "uy", "uz", "p"):
            assert np.array_equal(r.fields[k], f[k]), (r.id, k, np.max(np.abs(r.fields[k] - f[k])))
        assert r.mass_final == m_alone
        # the mass correction holds the order-parameter mass to the rounding
        # floor of the storage type over a few thousand sites
        assert abs(r.mass_final - r.mass0) <= (1e-12 if storage == "f64" else 1e-8) * abs(r.mass0)
        assert r.time_to_result >= r.t_done - r.t_admit >= 0.0


def test_admission_by_memory(require_gpu):
    """A reserve that leaves room for about one solve: never two at once."""
    import torch
    free, total = torch.cuda.mem_get_info(0)
    p, solid, init, W, _ = solve_spec(1)
    n = int(np.count_nonzero(solid == 0))
    per = 4 * 19 * 4 + 3 * 4 + 2 * 19 * 8 + 64
    nz, ny, nx = solid.shape
    one = (64 << 20) + n * per + 6 * 4 * (nx + 20) * (ny + 20) * (1 if nz == 1 else nz + 20)
    frac = max(0.0, (free - 1.5 * one) / total)
    srv = Server(storage="f32", hbm_reserve_frac=frac, chunk_steps=8)
    try:
        for k in range(4):
            srv.submit(k, p, solid, 16, init=init, init_width=W, want_fields=False)
        res = collect(srv, 4)
        st = srv.stats()
    finally:
        srv.close()
    assert len(res) == 4 and all(r.status == 0 for r in res)
    assert st["peak_active"] == 1


def test_convergence_retires_early(require_gpu):
    p, solid, init, W, _ = solve_spec(2)
    srv = Server(storage="f32", chunk_steps=10)
    try:
        srv.submit(0, p, solid, 100000, init=init, init_width=W, conv_tol=0.5, want_fields=False)
        res = collect(srv, 1)
    finally:
        srv.close()
    assert len(res) == 1 and res[0].status == 0
    assert res[0].steps_done < 100000


def test_stats_and_idle(require_gpu):
    specs = [solve_spec(k) for k in (3, 4)]
    srv = Server(storage="f32", chunk_steps=8)
    try:
        for k, (p, solid, init, W, steps) in enumerate(specs):
            srv.submit(k, p, solid, steps, init=init, init_width=W, want_fields=False)
        srv.wait_idle(300)
        st = srv.stats()
        res = srv.poll()
    finally:
        srv.close()
    assert st["completed"] == 2 and st["queued"] == 0 and st["active"] == 0
    sites = sum(int(np.count_nonzero(s[1] == 0)) * s[4] for s in specs)
    assert st["site_steps"] >= sites
    assert st["mlups_busy"] > 0 and st["ttr_p99"] >= st["ttr_p50"] > 0
    assert len(res) == 2


def test_served_solves_match_oracle(require_gpu):
    """Served FP64 solves, admitted while others run, against the FP64 oracle
    directly (the state the server builds from the slab description, then
    the reference driver loop with mass correction): fields within 1e-12."""
    from oracle.oracle_py import Oracle
    specs = [solve_spec(k) for k in (0, 1, 5)]
    srv = Server(storage="f64", max_active=2, chunk_steps=16)
    try:
        for k, (p, solid, init, W, steps) in enumerate(specs):
            srv.submit(k, p, solid, steps, init=init, init_width=W)
        res = collect(srv, len(specs))
    finally:
        srv.close()
    assert len(res) == len(specs)
    for r in res:
        assert r.status == 0, r.message
        p, solid, init, W, steps = specs[r.id]
        kind, a = init
        c = geometry.order_parameter(solid, "slab", W, origin=a[:3], axis=int(a[3]), thickness=a[4])
        h0, g0 = geometry.equilibrium(c, 1.0, p.rho0, p.rho1)
        o = Oracle(p, solid)
        o.upload_state(h0, g0)
        o.record_target_mass()
        o.run(steps, 0)
        fo = o.download()
        for k in ("c", "rho", "ux", "uy", "uz", "p"):
            d = float(np.max(np.abs(r.fields[k] - fo[k])))
            assert d <= 1e-12, (r.id, k, d)
        assert abs(r.mass_final - o.current_mass()) <= 1e-12 * abs(r.mass_final)
