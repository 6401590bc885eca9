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
    e = MultiPhaseGPU(in_place(case.params), case.solid)
    b = Batch()
    try:
        with pytest.raises(FeError):
            b.add(e)
    finally:
        b.free()
        e.free()
