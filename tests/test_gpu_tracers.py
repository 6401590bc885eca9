"""GPU tracers against the CPU restatement. The workload's bar: zero-
diffusivity trajectories to 1e-10 in FP64 against the FP64 oracle (here the
whole chain: CPU-oracle flow + numpy tracers vs engine + GPU tracers);
diffusive tracers match the restatement step for step on the engine's own
velocity (same Philox stream), and their dispersion matches 2 Dm t."""
import numpy as np
import pytest

from cases import make_case
from felbm_gpu_b200 import MultiPhaseGPU, geometry
from felbm_gpu_b200.tracers import Tracers, seed
from oracle import tracers_ref as tr
from oracle.oracle_py import Oracle
from parity import with_storage

pytestmark = pytest.mark.gpu


def flow_case(name="spheres_mrt"):
    # a stronger body force than the parity case, so tracers move
    return make_case(name, gx=2e-4) if name != "cyl2d_mrt" else make_case(name)


def grid(solid, f):
    nodes = geometry.site_nodes(solid)
    return tr.velocity_grid(solid.shape, nodes, f["ux"], f["uy"], f["uz"])


@pytest.mark.parametrize("order,substeps", [(2, 2), (1, 1)])
def test_tracers_match_restatement_on_engine_velocity(require_gpu, order, substeps):
    case = flow_case()
    e = MultiPhaseGPU(with_storage(case.params, "f64"), case.solid)
    try:
        e.upload_state(case.h0, case.g0)
        pos0, pid = seed(case.solid, 200, rng_seed=5)
        dm = np.where(np.arange(200) % 2 == 0, 0.0, 1e-3)
        ids = np.arange(200) + 1000
        t = Tracers(e, pos0, dm, ids=ids, substeps=substeps, order=order, rng_seed=99)
        pos = pos0.copy()
        for s in range(30):
            e.run(1)
            t.step()
            u = grid(case.solid, e.download())
            pos, vel = tr.step(pos, dm, ids, u, case.solid, s, substeps=substeps, order=order, seed=99)
        gp, gv = t.download()
        t.free()
    finally:
        e.free()
    assert np.max(np.abs(gp - pos)) <= 1e-10, np.max(np.abs(gp - pos))
    assert np.max(np.abs(gv - vel)) <= 1e-12
    assert np.max(np.abs(pos - pos0)) > 1e-3       # they moved


def test_zero_diffusivity_trajectories_match_fp64_oracle(require_gpu):
    """The full chain in FP64: oracle flow + restated tracers vs engine +
    GPU tracers, Dm = 0, 40 steps, <= 1e-10 (the workload's bound)."""
    case = flow_case()
    o = Oracle(case.params, case.solid)
    o.upload_state(case.h0, case.g0)
    e = MultiPhaseGPU(with_storage(case.params, "f64"), case.solid)
    try:
        e.upload_state(case.h0, case.g0)
        pos0, _ = seed(case.solid, 300, rng_seed=9)
        t = Tracers(e, pos0, 0.0, substeps=2, order=2)
        pos = pos0.copy()
        ids = np.arange(300)
        for s in range(40):
            e.run(1)
            t.step()
            o.step(1)
            pos, _ = tr.step(pos, np.zeros(300), ids, grid(case.solid, o.download()), case.solid, s, substeps=2)
        gp, _ = t.download()
        t.free()
    finally:
        e.free()
    assert np.max(np.abs(gp - pos)) <= 1e-10, np.max(np.abs(gp - pos))


def test_dispersion_statistics(require_gpu):
    """All fluid, no flow: variance 2 Dm t per axis (95 % band); 2-D lattices
    get no z motion."""
    solid = np.zeros((24, 24, 24), np.uint8)
    case = make_case("fluid_bgk")
    e = MultiPhaseGPU(with_storage(case.params, "f64"), solid)
    c = np.full(int(solid.size), 0.5)
    h0, g0 = geometry.equilibrium(c, 1.0, case.params.rho0, case.params.rho0)
    try:
        e.upload_state(h0, g0)
        n, dm, steps = 20000, 0.05, 30
        t = Tracers(e, np.full((3, n), 12.0), dm, substeps=2, rng_seed=4)
        for _ in range(steps):
            t.step()          # the state is at rest: velocity ~ 0
        p, _ = t.download()
        t.free()
    finally:
        e.free()
    var = ((p - 12.0) ** 2).mean(axis=1)
    assert np.all(np.abs(var / (2 * dm * steps) - 1.0) < 2.8 * np.sqrt(2.0 / n)), var


def test_2d_tracers_stay_in_plane(require_gpu):
    case = make_case("cyl2d_mrt")
    e = MultiPhaseGPU(with_storage(case.params, "f32"), case.solid)
    try:
        e.upload_state(case.h0, case.g0)
        pos0, _ = seed(case.solid, 100, rng_seed=2)
        t = Tracers(e, pos0, 0.01, rng_seed=3)
        for _ in range(10):
            e.run(1)
            t.step()
        p, _ = t.download()
        t.free()
    finally:
        e.free()
    assert np.all(p[2] == 0.0) and np.max(np.abs(p[:2] - pos0[:2])) > 0


def _cgrid(solid, f):
    nodes = geometry.site_nodes(solid)
    c = np.full(solid.size, np.nan)
    c[nodes] = f["c"]
    return c


def test_stretching_matches_restatement_on_engine_velocity(require_gpu):
    """Material line elements and the stretching rows (lambda, <log rho>,
    its variance, n_active, phase split) against the restatement, step for
    step on the engine's own velocity and order parameter, FP64, 1e-10."""
    case = make_case("spheres_mrt_wet", gx=2e-4)
    e = MultiPhaseGPU(with_storage(case.params, "f64"), case.solid)
    try:
        e.upload_state(case.h0, case.g0)
        n = 240
        pos0, _ = seed(case.solid, n, rng_seed=6)
        dm = np.where(np.arange(n) % 3 == 0, 2e-3, 0.0)
        ids = np.arange(n) + 7
        t = Tracers(e, pos0, dm, ids=ids, substeps=2, order=2, rng_seed=11, stretching=True, stretching_seed=77)
        rh, lr = t.stretch_state()
        assert np.max(np.abs(rh - tr.orientations(ids, 77))) <= 1e-13 and np.all(lr == 0.0)
        pos, rows = pos0.copy(), []
        for s in range(25):
            e.run(1)
            t.step()
            f = e.download()
            pos, _, rh, lr, row = tr.step(pos, dm, ids, grid(case.solid, f), case.solid, s, substeps=2, order=2,
                                          seed=11, stretch=(rh, lr), cgrid=_cgrid(case.solid, f))
            rows.append(row)
        got = t.stretch_rows()
        grh, glr = t.stretch_state()
        gp, _ = t.download()
        t.free()
    finally:
        e.free()
    want = np.array(rows)
    assert got.shape == want.shape
    assert np.array_equal(got[:, 0], np.arange(1, 26)) and np.array_equal(got[:, 4], want[:, 4])
    assert np.allclose(got, want, rtol=1e-9, atol=1e-12, equal_nan=True), np.nanmax(np.abs(got - want))
    assert np.all(got[:, 7] + got[:, 8] == got[:, 4])
    assert np.max(np.abs(gp - pos)) <= 1e-10
    assert np.max(np.abs(grh - rh)) <= 1e-10 and np.max(np.abs(glr - lr)) <= 1e-10
    assert np.max(np.abs(np.linalg.norm(grh, axis=0) - 1.0)) <= 1e-14
    assert np.max(np.abs(glr)) > 1e-6          # the elements stretched


def test_stretching_uniform_shear_exact_on_frozen_field(require_gpu):
    """A frozen analytic shear u = (g y, 0, 0): the line elements follow
    log|rho0 + t J rho0| to rounding; trajectories equal those without
    stretching bit for bit."""
    solid = np.zeros((8, 40, 40), np.uint8)
    case = make_case("fluid_bgk")
    e = MultiPhaseGPU(with_storage(case.params, "f64"), solid)
    gam = 0.01
    z, y, x = np.meshgrid(np.arange(8), np.arange(40), np.arange(40), indexing="ij")
    u = np.stack([(gam * y).reshape(-1), np.zeros(solid.size), np.zeros(solid.size)]).astype(np.float64)
    n = 64
    rng = np.random.default_rng(1)
    pos0 = np.stack([rng.uniform(5, 10, n), rng.uniform(8, 30, n), rng.uniform(2, 5, n)])
    try:
        t = Tracers(e, pos0, 0.0, substeps=3, order=1, stretching=True, stretching_seed=5)
        plain = Tracers(e, pos0, 0.0, substeps=3, order=1)
        rh0, _ = t.stretch_state()
        for tt in (t, plain):
            tt.set_velocity(u)
        for _ in range(20):
            t.step()
            plain.step()
        _, lr = t.stretch_state()
        p1, v1 = t.download()
        p2, v2 = plain.download()
        rows = t.stretch_rows(max_rows=8)
        rest = t.stretch_rows()
        t.free()
        plain.free()
    finally:
        e.free()
    J = np.array([[0, gam, 0], [0, 0, 0], [0, 0, 0]])
    want = np.log(np.linalg.norm(rh0 + 20 * (J @ rh0), axis=0))
    assert np.max(np.abs(lr - want)) < 1e-13
    assert np.array_equal(p1, p2) and np.array_equal(v1, v2)
    assert len(rows) == 8 and len(rest) == 12 and np.array_equal(np.r_[rows[:, 0], rest[:, 0]], np.arange(1, 21))
    assert np.all(rows[:, 4] == n) and np.all(np.isnan(rows[:, 5]))


def test_fused_snapshot_equals_refresh(require_gpu):
    """The first tracer set of an engine (velocity_skip 1) takes its velocity
    from the engine's next step; a second set refreshes the snapshot itself.
    Same tracers, same streams: identical trajectories and line elements, bit
    for bit, through solo steps, several steps at once and downloads."""
    case = flow_case("spheres_mrt_wet")
    e = MultiPhaseGPU(with_storage(case.params, "f32"), case.solid)
    try:
        e.upload_state(case.h0, case.g0)
        pos0, _ = seed(case.solid, 150, rng_seed=8)
        kw = dict(substeps=2, order=2, rng_seed=5, stretching=True)
        fused = Tracers(e, pos0, 1e-3, **kw)
        plain = Tracers(e, pos0, 1e-3, **kw)
        for s in range(12):
            e.run(1 if s % 4 else 3)
            fused.step()
            plain.step()
            if s == 6:
                assert np.array_equal(fused.download()[0], plain.download()[0])
        p1, v1 = fused.download()
        p2, v2 = plain.download()
        r1, r2 = fused.stretch_rows(), plain.stretch_rows()
        fused.free()
        plain.free()
    finally:
        e.free()
    assert np.array_equal(p1, p2) and np.array_equal(v1, v2)
    assert np.array_equal(r1, r2, equal_nan=True) and len(r1) == 12
