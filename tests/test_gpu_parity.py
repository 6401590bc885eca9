"""B200 engine vs the CPU oracle on the same seeded inputs (the reference's
compare_cpu_gpu design, src/compare_cpu_gpu.cu:244-294: identical initial
distributions, diff of h, g and of the macroscopic fields).

Tolerances (stated contract): FP64 storage max|dh|, max|dg|, and the fields
c, rho, u, p, mu <= 1e-12 after 100 steps; FP32 storage <= 1e-6 relative
(max|d| / max|ref|) after 20 steps, and after 100 steps no larger than the
error of the reference's own FP32 build (test_gpu_ref_kernels.py).
"""
import numpy as np
import pytest

from cases import CASES, make_case
from parity import maxdiff, reldiff, run_engine, run_oracle

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-6


@pytest.mark.parametrize("name", CASES)
def test_fp64_100_steps(require_gpu, name):
    case = make_case(name)
    h, g, f, st, nl = run_engine(case, 100, "f64")
    ho, go, fo, sto = run_oracle(case, 100)
    assert nl > 0
    assert maxdiff(h, ho) <= TOL64, maxdiff(h, ho)
    assert maxdiff(g, go) <= TOL64, maxdiff(g, go)
    for k in ("c", "rho", "ux", "uy", "uz", "p", "mu"):
        assert maxdiff(f[k], fo[k]) <= TOL64, (k, maxdiff(f[k], fo[k]))


@pytest.mark.parametrize("name", CASES)
def test_fp32_20_steps(require_gpu, name):
    """The reference's single-precision validation criterion: max|d| ~1e-6 on
    h and g after 20 steps (scripts/validate.sh:12-14; the metric is the
    max|delta| that compare_cpu_gpu prints, src/compare_cpu_gpu.cu:57-79).
    Longer runs are bounded against the reference's own FP32 kernels in
    test_gpu_ref_kernels.py."""
    case = make_case(name)
    h, g, f, _, _ = run_engine(case, 20, "f32")
    ho, go, fo, _ = run_oracle(case, 20)
    assert maxdiff(h, ho) <= TOL32, maxdiff(h, ho)
    assert maxdiff(g, go) <= TOL32, maxdiff(g, go)
    # macroscopic fields: the FP32 bound the workload states, max|dc| <= 1e-5
    for k in ("c", "rho", "p"):
        assert maxdiff(f[k], fo[k]) <= 1e-5, (k, maxdiff(f[k], fo[k]))


@pytest.mark.parametrize("name", ["spheres_mrt", "grf_mrt_mass", "openbnd_bgk"])
def test_step_api_matches_run(require_gpu, name):
    """fe_step + fe_apply_mass_correction (the reference driver's call pair)
    gives the same state as the fused fe_run loop."""
    case = make_case(name)
    h1, g1, _, _, _ = run_engine(case, 20, "f64", mode="step")
    h2, g2, _, _, _ = run_engine(case, 20, "f64", mode="run")
    assert maxdiff(h1, h2) <= 1e-14
    assert maxdiff(g1, g2) <= 1e-14


@pytest.mark.parametrize("name", ["spheres_mrt_wet", "grf_mrt_mass"])
def test_flow_stats(require_gpu, name):
    """Monitoring reductions (reference k_flow_stats) of the last step."""
    case = make_case(name)
    _, _, _, st, _ = run_engine(case, 30, "f64")
    _, _, _, sto = run_oracle(case, 30)
    assert np.allclose(st, sto, rtol=1e-10, atol=1e-14), (st, sto)


@pytest.mark.parametrize("storage,tol", [("f64", 1e-12), ("f32", 1e-8)])
def test_mass_correction_restores_target(require_gpu, storage, tol):
    """README.md:150-158: the correction restores the total order-parameter
    mass to M0 up to floating-point summation. Measured on the downloaded
    state (sum of h in FP64), after 50 and after 200 steps, so a drift that
    accumulates would show. The FP32 bound is the rounding floor of ~3.6k
    sites (each site's h rounded to FP32 after the injection)."""
    from felbm_gpu_b200 import MultiPhaseGPU
    from parity import with_storage
    case = make_case("grf_mrt_mass")
    e = MultiPhaseGPU(with_storage(case.params, storage), case.solid)
    try:
        e.upload_state(case.h0, case.g0)
        e.record_target_mass()
        m0 = e.get_target_mass()
        for steps in (50, 150):
            e.run(steps)
            h, _ = e.download_state()
            m = float(np.sum(h))
            assert abs(m - m0) / abs(m0) <= tol, (storage, steps, m, m0)
    finally:
        e.free()


def test_download_into_caller_buffers(require_gpu):
    """download_state(h, g) fills the caller's arrays with what a fresh
    download returns, on repeated calls; arrays of the wrong type, size or
    layout are refused."""
    from felbm_gpu_b200 import MultiPhaseGPU
    from parity import with_storage
    case = make_case("grf_mrt_mass")
    e = MultiPhaseGPU(with_storage(case.params, "f32"), case.solid)
    try:
        e.upload_state(case.h0, case.g0)
        hb, gb = np.full(e.Vn, np.nan), np.full(e.Vn, np.nan)
        for _ in range(2):
            e.run(3)
            h, g = e.download_state()
            h2, g2 = e.download_state(hb, gb)
            assert h2 is hb and g2 is gb
            assert np.array_equal(hb, h) and np.array_equal(gb, g)
        for bad in (np.empty(e.Vn, np.float32), np.empty(e.Vn - 1), np.empty(2 * e.Vn)[::2]):
            with pytest.raises(ValueError):
                e.download_state(bad, gb)
    finally:
        e.free()


@pytest.mark.parametrize("storage", ["f32", "f16g", "bf16s"])
def test_fp32_transfers_equal_fp64_transfers(require_gpu, storage, monkeypatch):
    """Large state transfers of the FP32-arithmetic storages move FP32 values
    (narrowed on the host before the copy up, widened after the copy down);
    FELBM_FP64_TRANSFERS=1 moves FP64 and converts on the device. Both give
    the same state and the same download, bit for bit, with and without a
    queued mass correction (64^3, above the size where the FP32 path starts)."""
    from felbm_gpu_b200 import MultiPhaseGPU, default_params, geometry
    solid, _ = geometry.grf((64, 64, 64), 4.0, 0.45, 5, flow_axis=0)
    p = default_params(use_mrt=1, use_halfway_bb=1, correct_op_mass=1, surface_tension=5e-3,
                       interface_width=4.0, gx=1e-5, storage=storage)
    rng = np.random.default_rng(3)

    def job(fp64):
        if fp64:
            monkeypatch.setenv("FELBM_FP64_TRANSFERS", "1")
        else:
            monkeypatch.delenv("FELBM_FP64_TRANSFERS", raising=False)
        e = MultiPhaseGPU(p, solid)
        try:
            assert e.Vn * 4 >= 4 << 20
            w = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
            h = (w[:, None] * c_fixed[None, :]).ravel()
            g = (w[:, None] * (1.0 + 0.01 * c_fixed[None, :])).ravel()
            e.upload_state(h, g)
            e.record_target_mass()
            e.run(3)
            out = [np.concatenate(e.download_state())]
            e.apply_mass_correction(want_drift=False)
            out.append(np.concatenate(e.download_state()))
            return out
        finally:
            e.free()

    e0 = MultiPhaseGPU(p, solid)
    n = e0.n
    e0.free()
    c_fixed = 0.5 + 0.5 * np.tanh(rng.standard_normal(n))
    a = job(False)
    b = job(True)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
