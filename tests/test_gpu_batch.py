"""Batches (fe_batch_*): many lattices advanced by one launch per pass. Every
member must get bit-for-bit the result it gets from fe_run alone (same
kernels, per-lattice control blocks and deterministic per-lattice
reductions), through membership changes and members stepped on their own
between batch runs."""
import numpy as np
import pytest

from cases import make_case
from felbm_gpu_b200 import Batch, MultiPhaseGPU
from parity import with_storage

pytestmark = pytest.mark.gpu

MIX = ["spheres_mrt", "cyl2d_mrt", "grf_mrt_mass", "grf_bgk_mass", "openbnd_bgk", "spheres_mrt_wet"]


def make_engine(name, storage):
    case = make_case(name)
    e = MultiPhaseGPU(with_storage(case.params, storage), case.solid)
    if case.open_bnd is not None:
        e.set_open_bnd(case.open_bnd)
    e.upload_state(case.h0, case.g0)
    if case.correct_mass:
        e.record_target_mass()
    return e


def alone(name, storage, steps):
    e = make_engine(name, storage)
    try:
        e.run(steps)
        h, g = e.download_state()
        return h, g, e.download(), e.flow_stats()
    finally:
        e.free()


@pytest.mark.parametrize("storage", ["f64", "f32", "f16s", "f16g"])
def test_batch_equals_alone(require_gpu, storage):
    steps = 23
    ref = {n: alone(n, storage, steps) for n in MIX}
    b = Batch()
    engines = {n: make_engine(n, storage) for n in MIX}
    try:
        for e in engines.values():
            b.add(e)
        assert b.size()[0] == len(MIX)
        b.run(10)
        b.run(13)
        for n, e in engines.items():
            h, g = e.download_state()
            f = e.download()
            hr, gr, fr, sr = ref[n]
            assert np.array_equal(h, hr), (n, np.max(np.abs(h - hr)))
            assert np.array_equal(g, gr), (n, np.max(np.abs(g - gr)))
            for k in ("c", "rho", "ux", "p", "mu"):
                assert np.array_equal(f[k], fr[k]), (n, k)
            assert np.array_equal(e.flow_stats(), sr), n
        assert b.launch_count() > 0
    finally:
        b.free()
        for e in engines.values():
            e.free()


def test_batch_membership_and_solo_steps(require_gpu):
    """Members join late, leave early, and one member is stepped on its own
    between batch runs; each still matches its own step count run alone."""
    storage = "f64"
    a = make_engine("spheres_mrt", storage)
    c = make_engine("grf_mrt_mass", storage)
    d = make_engine("cyl2d_mrt", storage)
    b = Batch()
    try:
        b.add(a)
        b.run(5)            # a: 5
        b.add(c)
        b.run(4)            # a: 9, c: 4
        c.run(3)            # c: 7 on its own
        b.add(d)
        b.run(6)            # a: 15, c: 13, d: 6
        b.remove(a)
        b.run(1)            # c: 14, d: 7
        for e, name, steps in ((a, "spheres_mrt", 15), (c, "grf_mrt_mass", 14), (d, "cyl2d_mrt", 7)):
            h, g = e.download_state()
            hr, gr, _, _ = alone(name, storage, steps)
            assert np.array_equal(h, hr), (name, np.max(np.abs(h - hr)))
            assert np.array_equal(g, gr), (name, np.max(np.abs(g - gr)))
    finally:
        b.free()
        for e in (a, c, d):
            e.free()


def test_batch_destroying_a_member(require_gpu):
    a = make_engine("spheres_mrt", "f32")
    c = make_engine("cyl2d_mrt", "f32")
    b = Batch()
    try:
        b.add(a)
        b.add(c)
        b.run(2)
        a.free()            # leaves the batch first
        b.members.remove(a)
        assert b.size()[0] == 1
        b.run(3)
        h, _ = c.download_state()
        hr, _, _, _ = alone("cyl2d_mrt", "f32", 5)
        assert np.array_equal(h, hr)
    finally:
        b.free()
        c.free()


def test_batch_rejects_mixed_storage(require_gpu):
    a = make_engine("spheres_mrt", "f32")
    c = make_engine("spheres_mrt", "f64")
    b = Batch()
    try:
        b.add(a)
        with pytest.raises(Exception, match="one storage type"):
            b.add(c)
    finally:
        b.free()
        a.free()
        c.free()


@pytest.mark.parametrize("storage", ["f64", "f32"])
def test_wide_offsets_agree_with_narrow(require_gpu, storage, monkeypatch):
    """The collide pass's 64-bit population offsets (taken for lattices whose
    arrays reach 2^32 entries; forced here at small size) address the same
    populations as the 32-bit variant: alone and in a batch, the states agree
    to rounding (the two instantiations may contract multiply-adds
    differently)."""
    steps = 17
    tol = 1e-12 if storage == "f64" else 2e-6
    ref = {n: alone(n, storage, steps) for n in MIX}
    monkeypatch.setenv("FELBM_WIDE_OFFSETS", "1")
    for n in MIX:
        h, g, f, s = alone(n, storage, steps)
        hr, gr, fr, sr = ref[n]
        d = max(np.max(np.abs(h - hr)), np.max(np.abs(g - gr)))
        assert d <= tol, (n, d)
        # the statistics are velocity means and maxima: FP32 rounding of
        # u ~ 0.05 leaves ~1e-7 noise on the near-zero components
        assert np.allclose(s, sr, rtol=1e-4, atol=tol if storage == "f64" else 2e-6), (n, s, sr)
    b = Batch()
    engines = {n: make_engine(n, storage) for n in MIX}
    try:
        for e in engines.values():
            b.add(e)
        b.run(steps)
        for n, e in engines.items():
            h, g = e.download_state()
            d = max(np.max(np.abs(h - ref[n][0])), np.max(np.abs(g - ref[n][1])))
            assert d <= tol, (n, d)
    finally:
        b.free()
        for e in engines.values():
            e.free()


@pytest.mark.parametrize("storage", ["f64", "f32"])
def test_two_rate_form_equals_general_transform(require_gpu, storage, monkeypatch):
    """MRT with one rate per moment parity (the reference's rate assignment)
    runs the closed two-rate form of M^-1 S M; FELBM_GENERAL_MRT=1 forces the
    19x15 transform. Both are the same linear map, so the states agree to
    rounding; cyl2d_mrt's explicit rates always take the general transform,
    and a batch mixing both forms gives every member its result alone."""
    steps = 23
    tol = 1e-12 if storage == "f64" else 2e-6
    names = ["spheres_mrt", "grf_mrt_mass", "spheres_mrt_wet"]
    fast = {n: alone(n, storage, steps) for n in names}
    monkeypatch.setenv("FELBM_GENERAL_MRT", "1")
    for n in names:
        h, g, _, _ = alone(n, storage, steps)
        d = max(np.max(np.abs(h - fast[n][0])), np.max(np.abs(g - fast[n][1])))
        assert 0 < d <= tol, (n, d)  # 0 would mean the switch changed nothing
    # engines made under FELBM_GENERAL_MRT=1 keep the general transform
    general = make_engine("grf_mrt_mass", storage)
    monkeypatch.delenv("FELBM_GENERAL_MRT")
    b = Batch()
    engines = {"general": general, "fast": make_engine("grf_mrt_mass", storage),
               "cyl2d_mrt": make_engine("cyl2d_mrt", storage)}
    try:
        monkeypatch.setenv("FELBM_GENERAL_MRT", "1")
        ref_general = alone("grf_mrt_mass", storage, steps)
        monkeypatch.delenv("FELBM_GENERAL_MRT")
        ref = {"general": ref_general, "fast": fast["grf_mrt_mass"], "cyl2d_mrt": alone("cyl2d_mrt", storage, steps)}
        for e in engines.values():
            b.add(e)
        b.run(steps)
        for n, e in engines.items():
            h, g = e.download_state()
            assert np.array_equal(h, ref[n][0]) and np.array_equal(g, ref[n][1]), n
    finally:
        b.free()
        for e in engines.values():
            e.free()


def test_batch_members_match_oracle(require_gpu):
    """Members of a mixed batch (porous MRT with mass correction, the 2-D
    cylinder pack on the general MRT transform, the open duct, wetting walls)
    against the FP64 oracle directly, 100 steps, at the FP64 parity bound."""
    from parity import maxdiff, run_oracle
    names = ["grf_mrt_mass", "cyl2d_mrt", "openbnd_bgk", "spheres_mrt_wet"]
    b = Batch()
    engines = {n: make_engine(n, "f64") for n in names}
    try:
        for e in engines.values():
            b.add(e)
        b.run(60)
        b.run(40)
        for n, e in engines.items():
            h, g = e.download_state()
            f = e.download()
            ho, go, fo, _ = run_oracle(make_case(n), 100)
            assert maxdiff(h, ho) <= 1e-12, (n, maxdiff(h, ho))
            assert maxdiff(g, go) <= 1e-12, (n, maxdiff(g, go))
            for k in ("c", "rho", "ux", "uy", "uz", "p", "mu"):
                assert maxdiff(f[k], fo[k]) <= 1e-12, (n, k, maxdiff(f[k], fo[k]))
    finally:
        b.free()
        for e in engines.values():
            e.free()
