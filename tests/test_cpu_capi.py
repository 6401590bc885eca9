"""The C-ABI library loads without a GPU, exports every symbol the header
declares, and rejects bad calls with a status instead of exiting."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from felbm_gpu_b200 import _capi, default_params, geometry

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "felbm_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(fe_[a-z0-9_]+)\s*\(", txt)))


def test_every_declared_symbol_is_exported():
    syms = header_symbols()
    assert len(syms) > 30
    missing = [s for s in syms if not hasattr(_capi.lib, s)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(header_symbols()) <= set(_capi.SIGNATURES)


def test_params_derivation_matches_reference():
    """kappa = 1.5 W sigma, beta = 12 sigma/W, mobility = coeff/beta,
    bnd_coeff = phi/kappa (reference compare_cpu_gpu.cu:115-118)."""
    p = default_params(interface_width=4.0, surface_tension=0.01, mobility_coeff=0.02, phi=0.003)
    assert abs(p.kappa - 1.5 * 4.0 * 0.01) < 1e-16
    assert abs(p.beta - 12 * 0.01 / 4.0) < 1e-16
    assert abs(p.mobility - 0.02 / p.beta) < 1e-16
    assert abs(p.bnd_coeff - 0.003 / p.kappa) < 1e-14
    assert p.mrt_lambda == 0.1875 and p.use_halfway_bb == 1 and p.storage == _capi.FE_F64
    # reference rate assignment: q and m magic, the others follow s0
    assert list(p.mrt_rate_mode)[1:] == [0, 0, 1, 0, 0, 1]


def test_errors_are_status_codes():
    assert _capi.lib.fe_engine_destroy(None) == 0
    p = default_params()
    h = C.c_void_p()
    rc = _capi.lib.fe_engine_create(C.byref(p), 0, 4, 4, None, -1, C.byref(h))
    assert rc == _capi.FE_ERR_ARG
    assert b"bad arguments" in _capi.lib.fe_last_error()
    assert _capi.lib.fe_step(None, 1) == _capi.FE_ERR_ARG
    assert _capi.lib.fe_version().startswith(b"felbm_b200")


def test_engine_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        return
    p = default_params()
    solid = np.zeros((4, 4, 4), np.uint8)
    h = C.c_void_p()
    rc = _capi.lib.fe_engine_create(C.byref(p), 4, 4, 4, solid.ctypes.data_as(C.POINTER(C.c_uint8)), -1,
                                    C.byref(h))
    assert rc == _capi.FE_ERR_NO_DEVICE


def test_geometry_generators_are_seeded():
    a, pa = geometry.grf((24, 24, 24), 3.0, 0.4, 11)
    b, pb = geometry.grf((24, 24, 24), 3.0, 0.4, 11)
    c, _ = geometry.grf((24, 24, 24), 3.0, 0.4, 12)
    assert (a == b).all() and pa == pb and not (a == c).all()
    assert 0.3 < pa <= 0.4
    m, por = geometry.cylinders((1, 200, 200), 6.0, 12.0, 0.65, 12345)
    assert abs(por - 0.65) < 0.03


def test_grf_keeps_one_percolating_cluster():
    from scipy import ndimage
    m, _ = geometry.grf((32, 32, 32), 3.0, 0.35, 5, flow_axis=0, open_flow=True)
    fluid = m == 0
    lab, nlab = ndimage.label(fluid, structure=np.ones((3, 3, 3)))
    assert nlab >= 1
    # one cluster (periodic links may merge labels scipy sees as separate)
    xs = np.where(fluid.any(axis=(0, 1)))[0]
    assert xs.min() == 0 and xs.max() == 31


def test_open_padding_and_lists():
    medium = np.zeros((6, 5, 10), np.uint8)
    medium[2, 2, 0] = 1
    s = geometry.pad_open(medium, 0, 2, 2)
    assert s.shape == (6, 5, 18)
    assert s[:, :, :4].sum() == 0 and s[:, :, -4:].sum() == 0
    inl, outl, bv, br, coord = geometry.open_lists(s, 0, 2, split_axis=1)
    assert len(inl) == 30 and len(outl) == 30 and len(bv) == 120 and len(br) == 120
    nodes = geometry.site_nodes(s)
    xs = nodes % 18
    assert (xs[inl] == 2).all() and (xs[outl] == 15).all()
    assert set(xs[br]) == {2, 15}


def test_equilibrium_moments():
    m = np.zeros((3, 4, 5), np.uint8)
    c = np.linspace(0, 1, 60)
    h, g = geometry.equilibrium(c, 0.7, 2.0, 1.0)
    assert np.allclose(h.reshape(19, -1).sum(0), c, atol=1e-15)
    assert np.allclose(g.reshape(19, -1).sum(0), 0.7, atol=1e-15)
    del m


def _order_parameter_np(solid, kind, width, a):
    """The initial order parameter per site in node order, restated with
    numpy: slab of thickness a[4] from a[axis] along axis a[3] (periodic),
    droplet of radius a[3] at a[0:3] (periodic), or uniform a[0]."""
    nz, ny, nx = solid.shape
    z, y, x = np.nonzero(solid == 0)
    pos = [x.astype(np.float64), y.astype(np.float64), z.astype(np.float64)]
    N = [nx, ny, nz]
    if kind == 0:
        return np.full(x.size, a[0])
    if kind == 1:
        ax = int(a[3])
        L, T = float(N[ax]), a[4]
        sd = np.fmod(pos[ax] - a[ax], L)
        sd = np.where(sd < 0, sd + L, sd)
        u = sd + 0.5
        d = np.where(u < T, np.minimum(u, T - u), -np.minimum(u - T, L - u))
    else:
        r2 = np.zeros(x.size)
        for q in range(3):
            dd = np.abs(pos[q] - a[q])
            dd = np.minimum(dd, N[q] - dd)
            r2 += dd * dd
        d = a[3] - np.sqrt(r2)
    return 0.5 * (1.0 + np.tanh(2.0 * d / width))


@pytest.mark.parametrize("shape", [(9, 7, 13), (1, 40, 33), (6, 1, 1), (12, 12, 12)])
def test_initial_order_parameter(shape):
    """fe_init_order_parameter (rows filled in parallel from per-row site
    counts) against a numpy restatement: site order and values, for the
    uniform, slab (each axis) and droplet fields on a random mask."""
    rng = np.random.default_rng(sum(shape))
    solid = (rng.random(shape) < 0.4).astype(np.uint8)
    nz, ny, nx = shape
    runs = [("uniform", 0, dict(c=0.3), [0.3, 0, 0, 0, 0]),
            ("droplet", 2, dict(centre=(nx / 2, ny / 3, nz / 4), radius=3.0), [nx / 2, ny / 3, nz / 4, 3.0, 0])]
    for ax in range(3):
        o = (1.5, 2.0, 0.5)
        runs.append(("slab", 1, dict(origin=o, axis=ax, thickness=[nx, ny, nz][ax] / 3.0),
                     [o[0], o[1], o[2], float(ax), [nx, ny, nz][ax] / 3.0]))
    for name, kind, kw, a in runs:
        c = geometry.order_parameter(solid, name, 4.0, **kw)
        want = _order_parameter_np(solid, kind, 4.0, a)
        assert c.shape == want.shape
        assert np.max(np.abs(c - want), initial=0.0) <= 1e-15, (name, a)


def test_autotune_table_round_trip(tmp_path):
    """The autotune table's text form: loaded entries are saved back as read;
    a malformed file is refused."""
    from felbm_gpu_b200.engine import tune_clear, tune_load, tune_save
    p = tmp_path / "tune.txt"
    rows = ["0 1 1 1 7 23 3 8", "1 1 1 1 12 16 2 32"]
    p.write_text("# a table\n" + "\n".join(rows) + "\n")
    tune_clear()
    tune_load(str(p))
    q = tmp_path / "out.txt"
    tune_save(str(q))
    got = [l for l in q.read_text().splitlines() if not l.startswith("#")]
    assert sorted(got) == sorted(rows)
    p.write_text("0 1 1 1 7 23 9 8\n")
    import pytest
    from felbm_gpu_b200._capi import FeError
    with pytest.raises(FeError):
        tune_load(str(p))
    tune_clear()
