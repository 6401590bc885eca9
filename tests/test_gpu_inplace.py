"""The in-place population layout (FE_POP_IN_PLACE: one buffer, the two
phases of the AA pattern) against the FP64 oracle and against the
two-buffer layout.

Tolerances: FP64 max|dh|, max|dg| and the fields c, rho, u, p, mu <= 1e-12
after an even (100) and an odd (99) step count, so the state is read back
from both phases; FP32 without mass correction bit-equal to the two-buffer
layout (the same arithmetic per site), with mass correction within 1e-6 (the
mass sums are added per brick instead of per chunk in one of the phases).
"""
import numpy as np
import pytest

from cases import make_case
from felbm_gpu_b200 import Batch, MultiPhaseGPU
from felbm_gpu_b200._capi import FeError
from parity import maxdiff, run_oracle, with_storage

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
FIELDS = ("c", "rho", "ux", "uy", "uz", "p", "mu")


def in_place(params, storage="f64"):
    p = with_storage(params, storage)
    p.pop_layout = 1
    return p


def run_in_place(case, steps, storage="f64", mode="run", layout=1):
    p = with_storage(case.params, storage)
    p.pop_layout = layout
    e = MultiPhaseGPU(p, case.solid)
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
        f = e.download()
        return h, g, f
    finally:
        e.free()


def assert_fp64(h, g, f, ho, go, fo, tag):
    assert maxdiff(h, ho) <= TOL64, (tag, "h", maxdiff(h, ho))
    assert maxdiff(g, go) <= TOL64, (tag, "g", maxdiff(g, go))
    for k in FIELDS:
        assert maxdiff(f[k], fo[k]) <= TOL64, (tag, k, maxdiff(f[k], fo[k]))


@pytest.mark.parametrize("steps", [99, 100])
@pytest.mark.parametrize("name", ["fluid_mrt", "spheres_bgk", "spheres_mrt_wet", "cyl2d_mrt", "grf_mrt_mass",
                                  "openbnd_mrt_buf"])
def test_in_place_fp64_vs_oracle(require_gpu, name, steps):
    case = make_case(name)
    h, g, f = run_in_place(case, steps)
    ho, go, fo, _ = run_oracle(case, steps)
    assert_fp64(h, g, f, ho, go, fo, (name, steps))


def test_in_place_step_loop_and_reads_between_steps(require_gpu):
    """fe_step one at a time with the mass correction, the state and the
    fields read back after odd and even steps (each read from the swapped
    phase turns the state into the standard layout first), then more steps;
    against the oracle's loop."""
    case = make_case("grf_mrt_mass")
    e = MultiPhaseGPU(in_place(case.params), case.solid)
    o = None
    try:
        e.upload_state(case.h0, case.g0)
        e.record_target_mass()
        from oracle.oracle_py import Oracle
        o = Oracle(case.params, case.solid)
        o.upload_state(case.h0, case.g0)
        o.record_target_mass()
        for block in (7, 6, 1, 30):
            for _ in range(block):
                e.step(1)
                e.apply_mass_correction(want_drift=False)
                o.step(1)
                o.apply_mass_correction()
            h, g = e.download_state()
            f = e.download()
            ho, go = o.download_state()
            fo = o.download()
            assert_fp64(h, g, f, ho, go, fo, block)
    finally:
        e.free()


@pytest.mark.parametrize("steps", [20, 21])
def test_in_place_fp32_equals_two_buffers(require_gpu, steps):
    case = make_case("spheres_mrt_wet")
    h1, g1, f1 = run_in_place(case, steps, "f32", layout=1)
    h0, g0, f0 = run_in_place(case, steps, "f32", layout=0)
    assert np.array_equal(h1, h0) and np.array_equal(g1, g0)
    for k in FIELDS:
        assert np.array_equal(f1[k], f0[k]), k


def test_in_place_fp32_mass_correction(require_gpu):
    case = make_case("grf_mrt_mass")
    h1, g1, _ = run_in_place(case, 41, "f32", layout=1)
    h0, g0, _ = run_in_place(case, 41, "f32", layout=0)
    assert maxdiff(h1, h0) <= 1e-6 and maxdiff(g1, g0) <= 1e-6
    m0 = float(np.sum(case.h0))
    assert abs(float(np.sum(h1)) - m0) / abs(m0) <= 1e-8


def test_in_place_holds_one_buffer(require_gpu):
    import torch
    case = make_case("c2_open_mrt")
    warm = make_case("spheres_bgk")  # loads the set-up kernels before measuring
    MultiPhaseGPU(with_storage(warm.params, "f32"), warm.solid).free()
    before = torch.cuda.mem_get_info(0)[0]
    e0 = MultiPhaseGPU(with_storage(case.params, "f32"), case.solid)
    mid = torch.cuda.mem_get_info(0)[0]
    e1 = MultiPhaseGPU(in_place(case.params, "f32"), case.solid)
    after = torch.cuda.mem_get_info(0)[0]
    try:
        two, one = before - mid, mid - after
        pops = 2 * 19 * 4 * (case.h0.size // 19)  # one buffer of h and g
        assert two - one >= 0.9 * pops, (two, one, pops)
    finally:
        e1.free()
        e0.free()


def test_in_place_refused_where_unsupported(require_gpu):
    case = make_case("spheres_bgk")
    with pytest.raises(FeError):
        MultiPhaseGPU(in_place(case.params, "f16g"), case.solid)


def test_batch_with_in_place_members_vs_oracle(require_gpu):
    """A batch of in-place members of two brick shapes (3-D porous with mass
    correction, the 2-D cylinder pack) beside a two-buffer member: odd step
    counts, a state read between the runs (which swaps that member back to
    the standard layout and makes the batch rebuild), each member against
    the FP64 oracle after 63 steps."""
    from parity import run_oracle
    names = {"grf_mrt_mass": 1, "cyl2d_mrt": 1, "spheres_mrt_wet": 0}
    engines = {}
    b = Batch()
    try:
        for n, layout in names.items():
            case = make_case(n)
            p = with_storage(case.params, "f64")
            p.pop_layout = layout
            e = MultiPhaseGPU(p, case.solid)
            e.upload_state(case.h0, case.g0)
            if case.correct_mass:
                e.record_target_mass()
            engines[n] = e
            b.add(e)
        b.run(37)
        engines["grf_mrt_mass"].download_state()
        b.run(26)
        for n, e in engines.items():
            h, g = e.download_state()
            f = e.download()
            ho, go, fo, _ = run_oracle(make_case(n), 63)
            assert_fp64(h, g, f, ho, go, fo, n)
    finally:
        b.free()
        for e in engines.values():
            e.free()


def test_served_in_place_equals_alone(require_gpu):
    """The request loop with every solve in place: each result bit-for-bit
    the same solve run alone in place."""
    import time
    from felbm_gpu_b200 import geometry
    from felbm_gpu_b200.serving import Server
    from test_gpu_serving import collect, solve_spec
    specs = [solve_spec(k) for k in range(6)]
    srv = Server(storage="f32", max_active=3, chunk_steps=16, pop_layout="in_place")
    try:
        for k, (p, solid, init, W, steps) in enumerate(specs):
            srv.submit(k, p, solid, steps, init=init, init_width=W)
            time.sleep(0.01)
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
        e = MultiPhaseGPU(in_place(p, "f32"), solid)
        try:
            e.upload_state(h0, g0)
            e.record_target_mass()
            e.run(steps)
            f = e.download()
            m = e.current_mass()
        finally:
            e.free()
        for k in ("c", "rho", "ux", "uy", "uz", "p"):
            assert np.array_equal(r.fields[k], f[k]), (r.id, k, np.max(np.abs(r.fields[k] - f[k])))
        assert r.mass_final == m


def test_in_place_tracers_and_checkpoint_equal_two_buffers(require_gpu, tmp_path):
    """Tracers on an in-place engine (the fused snapshot of the next step and
    the explicit refresh pass from either phase) and a checkpoint written
    after an odd step count: trajectories, line elements and the restarted
    run bit-equal to the two-buffer engine's (FP32, no mass correction)."""
    from felbm_gpu_b200 import files
    from felbm_gpu_b200.tracers import Tracers, seed
    case = make_case("spheres_mrt_wet")
    pos0, _ = seed(case.solid, 150, rng_seed=8)
    kw = dict(substeps=2, order=2, rng_seed=5, stretching=True)
    out = {}
    for layout in (0, 1):
        p = with_storage(case.params, "f32")
        p.pop_layout = layout
        e = MultiPhaseGPU(p, case.solid)
        try:
            e.upload_state(case.h0, case.g0)
            fused = Tracers(e, pos0, 1e-3, **kw)
            plain = Tracers(e, pos0, 1e-3, **kw)
            for s in range(9):
                e.run(1 if s % 4 else 3)
                fused.step()
                plain.step()
            pf, vf = fused.download()
            pp, vp = plain.download()
            fused.free()
            plain.free()
            ck = str(tmp_path / f"ck{layout}.h5")
            files.write_checkpoint(e, ck, 15)
            e.run(5)
            h, g = e.download_state()
        finally:
            e.free()
        r = MultiPhaseGPU(p, case.solid)  # restart from the checkpoint
        try:
            assert files.read_checkpoint(r, ck) == 15
            r.run(5)
            hr, gr = r.download_state()
        finally:
            r.free()
        assert np.array_equal(hr, h) and np.array_equal(gr, g)
        out[layout] = (pf, vf, pp, vp, h, g)
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b, equal_nan=True)


@pytest.mark.parametrize("brick", ["8x8x8", "8x8x4"])
def test_in_place_other_bricks_vs_oracle(require_gpu, brick):
    """The in-place phases on the other brick shapes (their halo-1 tiles of
    population bases differ), 37 steps (the state read back from phase 1)."""
    from felbm_gpu_b200 import _capi
    case = make_case("grf_mrt_mass")
    p = in_place(case.params)
    p.brick = _capi.BRICK[brick]
    e = MultiPhaseGPU(p, case.solid)
    try:
        e.upload_state(case.h0, case.g0)
        e.record_target_mass()
        e.run(37)
        h, g = e.download_state()
        f = e.download()
    finally:
        e.free()
    ho, go, fo, _ = run_oracle(case, 37)
    assert_fp64(h, g, f, ho, go, fo, brick)


def test_in_place_refused_with_wide_offsets(require_gpu, monkeypatch):
    """Lattices that need 64-bit population offsets keep two buffers (the
    in-place passes address populations with 32-bit bases)."""
    monkeypatch.setenv("FELBM_WIDE_OFFSETS", "1")
    case = make_case("spheres_bgk")
    with pytest.raises(FeError):
        MultiPhaseGPU(in_place(case.params), case.solid)
