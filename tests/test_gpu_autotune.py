"""Autotuned layouts: every 3-D brick (8x8x8, 8x8x4, 16x8x8; the default is
16x8x8 for FP64/FP32) meets the same parity bar against the FP64 oracle;
the steps per graph launch change nothing in the result; fe_autotune times every
candidate, records the fastest for the size class, and engines created with
brick "auto" in that class take it; a batch mixing bricks gives every
member its result alone."""
import ctypes as C

import numpy as np
import pytest

from cases import make_case
from felbm_gpu_b200 import Batch, MultiPhaseGPU, _capi, geometry
from felbm_gpu_b200.engine import autotune, default_params, tune_clear
from parity import maxdiff, run_oracle, with_storage

pytestmark = pytest.mark.gpu

CASES3D = ["spheres_mrt", "spheres_mrt_wet", "grf_mrt_mass", "grf_bgk_mass", "openbnd_bgk", "openbnd_mrt_buf"]


def _params(case, storage, brick="auto", graph_steps=0):
    p = with_storage(case.params, storage)
    p.brick = _capi.BRICK[brick]
    p.graph_steps = graph_steps
    return p


def _run(case, storage, steps, brick="auto", graph_steps=0):
    e = MultiPhaseGPU(_params(case, storage, brick, graph_steps), case.solid)
    try:
        if case.open_bnd is not None:
            e.set_open_bnd(case.open_bnd)
        e.upload_state(case.h0, case.g0)
        if case.correct_mass:
            e.record_target_mass()
        e.run(steps)
        h, g = e.download_state()
        return h, g, e.download(), e.layout()
    finally:
        e.free()


@pytest.mark.parametrize("brick", ["8x8x8", "8x8x4", "16x8x8"])
@pytest.mark.parametrize("name", CASES3D)
def test_alternative_bricks_fp64_parity(require_gpu, name, brick):
    case = make_case(name)
    h, g, f, lay = _run(case, "f64", 100, brick)
    assert lay == (brick, 2)
    ho, go, fo, _ = run_oracle(case, 100)
    assert maxdiff(h, ho) <= 1e-12 and maxdiff(g, go) <= 1e-12, (maxdiff(h, ho), maxdiff(g, go))
    for k in ("c", "rho", "ux", "p", "mu"):
        assert maxdiff(f[k], fo[k]) <= 1e-12, k


@pytest.mark.parametrize("brick", ["8x8x8", "8x8x4"])
def test_alternative_bricks_fp32(require_gpu, brick):
    case = make_case("grf_mrt_mass")
    h, g, _, _ = _run(case, "f32", 20, brick)
    h8, g8, _, _ = _run(case, "f32", 20, "16x8x8")
    assert maxdiff(h, h8) <= 1e-6 and maxdiff(g, g8) <= 1e-6


def test_graph_steps_do_not_change_the_result(require_gpu):
    case = make_case("spheres_mrt_wet")
    ref = _run(case, "f32", 37, "8x8x8", 2)
    for gs in (1, 5, 8, 32):
        h, g, _, lay = _run(case, "f32", 37, "8x8x8", gs)
        assert lay == ("8x8x8", gs)
        assert np.array_equal(h, ref[0]) and np.array_equal(g, ref[1]), gs


def test_autotune_choice_is_taken(require_gpu):
    tune_clear()
    solid, _ = geometry.grf((48, 48, 48), 4.0, 0.45, 3, flow_axis=0)
    p = default_params(use_mrt=1, storage="f32", correct_op_mass=1)
    rep = autotune(p, solid, steps=6)
    assert len(rep["candidates"]) == 5 and all(m > 0 for _, _, m in rep["candidates"])
    best = max(rep["candidates"], key=lambda c: c[2])
    assert (rep["brick"], rep["graph_steps"]) == best[:2]
    e = MultiPhaseGPU(p, solid)
    try:
        assert e.layout() == (rep["brick"], rep["graph_steps"])
    finally:
        e.free()
    # another size class keeps the default (16x8x8 for FP32)
    small, _ = geometry.grf((20, 20, 20), 4.0, 0.45, 3, flow_axis=0)
    e = MultiPhaseGPU(p, small)
    try:
        assert e.layout() == ("16x8x8", 2)
    finally:
        e.free()
    tune_clear()


def test_batch_mixing_bricks_equals_alone(require_gpu):
    case = make_case("grf_mrt_mass")
    bricks = ["8x8x8", "8x8x4", "16x8x8"]
    ref = {b: _run(case, "f32", 15, b)[:2] for b in bricks}
    b = Batch()
    engines = {}
    try:
        for br in bricks:
            e = MultiPhaseGPU(_params(case, "f32", br), case.solid)
            e.upload_state(case.h0, case.g0)
            e.record_target_mass()
            engines[br] = e
            b.add(e)
        b.run(15)
        for br, e in engines.items():
            h, g = e.download_state()
            assert np.array_equal(h, ref[br][0]) and np.array_equal(g, ref[br][1]), br
    finally:
        b.free()
        for e in engines.values():
            e.free()


def test_bricks_refused_where_not_built(require_gpu):
    case = make_case("spheres_mrt")
    with pytest.raises(_capi.FeError, match="FP64 and FP32"):
        MultiPhaseGPU(_params(case, "f16g", "8x8x4"), case.solid)
    c2 = make_case("cyl2d_mrt")
    with pytest.raises(_capi.FeError, match="16x16x1"):
        MultiPhaseGPU(_params(c2, "f32", "8x8x8"), c2.solid)


@pytest.mark.parametrize("storage", ["f16g", "f16s", "bf16g"])
def test_16bit_storages_on_wide_bricks(require_gpu, storage):
    """16x8x8 bricks for the 16-bit storages: the same per-site arithmetic as
    on 8x8x8 (only the order of the mass and statistics sums differs)."""
    case = make_case("grf_mrt_mass")
    h, g, _, lay = _run(case, storage, 20, "16x8x8")
    h8, g8, _, _ = _run(case, storage, 20, "8x8x8")
    assert lay == ("16x8x8", 2)
    assert maxdiff(h, h8) <= 2e-3 and maxdiff(g, g8) <= 2e-3, (maxdiff(h, h8), maxdiff(g, g8))
