"""CPU tests of the oracle: invariants the reference documents, its own
self-checks, and (when present) the golden vectors produced by the
reference's kernels."""
import glob
import os

import numpy as np
import pytest

from cases import make_case
from felbm_gpu_b200 import default_params, geometry
from oracle.oracle_py import Oracle, mrt_matrices

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_mrt_basis_orthogonal_and_inverse():
    M, Minv = mrt_matrices()
    assert np.abs(M @ Minv - np.eye(19)).max() < 1e-14
    D = (M * M).sum(1)
    assert np.abs(M @ M.T - np.diag(D)).max() == 0
    # d'Humieres et al. (2002) D3Q19 row norms
    assert list(D.astype(int)) == [19, 2394, 252, 10, 40, 10, 40, 10, 40, 36, 72, 12, 24, 4, 4, 4, 8, 8, 8]


def test_inplace_program_equals_gather():
    """multiphase_gpu.cuh:245-282: the in-place op program reproduces the
    gather streaming; here over 20 full steps, bit for bit."""
    case = make_case("spheres_mrt")
    a = Oracle(case.params, case.solid)
    b = Oracle(case.params, case.solid, inplace=True)
    counts = b.inplace_counts()
    assert counts[0] > 0 and counts[1] == 0 and counts[2] == 0
    for o in (a, b):
        o.upload_state(case.h0, case.g0)
        o.step(20)
    ha, ga = a.download_state()
    hb, gb = b.download_state()
    assert np.array_equal(ha, hb) and np.array_equal(ga, gb)


def test_rest_state_is_a_fixed_point():
    """Uniform c and p at rest without force: the equilibrium is stationary."""
    solid = geometry.spheres((12, 12, 12), 2.5, 3, 2.0, 3)
    p = default_params(use_mrt=1, rho0=3.0, rho1=1.0)
    n = int((solid == 0).sum())
    h, g = geometry.equilibrium(np.full(n, 0.3), 1.0, p.rho0, p.rho1)
    o = Oracle(p, solid)
    o.upload_state(h, g)
    o.step(10)
    h2, g2 = o.download_state()
    assert np.abs(h2 - h).max() < 1e-15 and np.abs(g2 - g).max() < 1e-15


def test_mass_correction_invariants():
    """README.md:150-163: the correction restores M0 exactly (up to summation)
    and adds no momentum (sum_k w_k e_k = 0)."""
    case = make_case("grf_mrt_mass")
    o = Oracle(case.params, case.solid)
    o.upload_state(case.h0, case.g0)
    o.record_target_mass()
    m0 = o.get_target_mass()
    o.step(5)
    h_before, g_before = o.download_state()
    drift = o.apply_mass_correction()
    assert drift != 0.0
    h_after, g_after = o.download_state()
    assert abs(o.current_mass() - m0) <= 1e-12 * abs(m0)
    n = o.n
    dh = (h_after - h_before).reshape(19, n)
    ex = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1])
    # zero first moment up to the rounding of h (|h| < 1): ~19 ulp of h
    assert np.abs(ex @ dh).max() < 1e-15
    assert np.array_equal(g_after, g_before)


def test_long_run_is_finite():
    case = make_case("cyl2d_mrt")
    o = Oracle(case.params, case.solid)
    o.upload_state(case.h0, case.g0)
    o.step(200)
    h, g = o.download_state()
    assert np.isfinite(h).all() and np.isfinite(g).all()


def test_tables_on_a_wall():
    """Near-wall cases of the reference builders on a hand-checked site: a
    fluid node with a solid neighbour at +x and fluid at -x, -2x."""
    solid = np.zeros((1, 1, 8), np.uint8)
    solid[0, 0, 5] = 1
    p = default_params(use_halfway_bb=1)
    o = Oracle(p, solid)
    n = o.n
    i = 4                      # node x = 4 (sites are x = 0..4, 6, 7)
    m = 1                      # +x
    cdm, cdp = o.table(0), o.table(1)
    bcase, bc1 = o.table(2), o.table(3)
    lcase, lc1 = o.table(5), o.table(6)
    idx = (m - 1) * n + i
    assert (cdm[idx], cdp[idx]) == (3, 4)          # backward pair (x-1, x)
    assert bcase[idx] == 4 and bc1[idx] == 3       # 2-point backward, bounce-back
    assert lcase[idx] == 3 and lc1[idx] == 3       # one-sided BB Laplacian
    src = o.table(9)
    assert src[1 * n + 5] == 2 * n + 5             # +x at x=6: x=5 is solid -> own -x slot
    assert src[2 * n + i] == 1 * n + i             # -x at x=4 comes from solid x=5: own +x slot


@pytest.mark.skipif(not glob.glob(os.path.join(GOLDEN, "*.npz")), reason="no golden vectors committed")
@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))))
def test_oracle_matches_reference_golden(path):
    """Golden vectors: the reference's own kernels (device_engine.cuh on sm_100a,
    FP64) after 20 steps, generated by tests/golden/make_golden.py."""
    d = np.load(path)
    name = str(d["case"])
    kw = {k[3:]: d[k].item() for k in d.files if k.startswith("kw_")}
    case = make_case(name, **kw)
    o = Oracle(case.params, case.solid)
    if case.open_bnd is not None:
        o.set_open_bnd(case.open_bnd)
    o.upload_state(case.h0, case.g0)
    if case.correct_mass:
        o.record_target_mass()
    o.run(int(d["steps"]), 0)
    h, g = o.download_state()
    f = o.fields()
    sel = d["sel"]
    assert np.abs(h[sel] - d["h"]).max() <= 1e-13
    assert np.abs(g[sel] - d["g"]).max() <= 1e-13
    assert abs(h.sum() - float(d["h_sum"])) <= 1e-10 and abs(g.sum() - float(d["g_sum"])) <= 1e-10
    sites = d["sites"] if "sites" in d.files else np.arange(o.n)
    for k in ("c", "rho", "ux", "uy", "uz", "p", "mu"):
        assert np.abs(f[k][sites] - d["f_" + k]).max() <= 1e-13, k
