"""Checkpoint and field files on the GPU engine: a run continued from a
checkpoint equals the uninterrupted run bit for bit (the reference's claim
for its double build, README "checkpoint"), the original M0 is kept, a
checkpoint of another geometry is refused, and a field file holds what
fe_download_fields returns."""
import numpy as np
import pytest

from cases import make_case
from felbm_gpu_b200 import MultiPhaseGPU, files
from parity import with_storage

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("storage", ["f64", "f32"])
def test_checkpoint_restart_is_exact(require_gpu, tmp_path, storage):
    case = make_case("grf_mrt_mass")
    p = str(tmp_path / "checkpoint.h5")
    a = MultiPhaseGPU(with_storage(case.params, storage), case.solid)
    b = MultiPhaseGPU(with_storage(case.params, storage), case.solid)
    try:
        a.upload_state(case.h0, case.g0)
        a.record_target_mass()
        m0 = a.get_target_mass()
        a.run(15)
        files.write_checkpoint(a, p, 15)
        a.run(10)
        h1, g1 = a.download_state()
        assert files.read_checkpoint(b, p) == 15
        assert b.get_target_mass() == m0
        b.set_time(15)
        b.run(10)
        h2, g2 = b.download_state()
    finally:
        a.free()
        b.free()
    # FP64 on disk holds FP32 populations exactly, so both storages restart exactly
    assert np.array_equal(h1, h2) and np.array_equal(g1, g2)


def test_checkpoint_of_other_geometry_is_refused(require_gpu, tmp_path):
    a = make_case("spheres_mrt")
    c = make_case("cyl2d_mrt")
    p = str(tmp_path / "ck.h5")
    ea = MultiPhaseGPU(a.params, a.solid)
    ec = MultiPhaseGPU(c.params, c.solid)
    try:
        ea.upload_state(a.h0, a.g0)
        files.write_checkpoint(ea, p, 1)
        with pytest.raises(Exception, match="geometry mismatch"):
            files.read_checkpoint(ec, p)
    finally:
        ea.free()
        ec.free()


@pytest.mark.parametrize("f32,deflate", [(False, 0), (True, 0), (False, 4), (True, 9)])
def test_field_file_matches_download(require_gpu, tmp_path, f32, deflate):
    """output_float32 / output_deflate (gzip level, one chunk per dataset)."""
    case = make_case("spheres_mrt_wet")
    p = str(tmp_path / "fields_20.h5")
    e = MultiPhaseGPU(case.params, case.solid)
    try:
        e.upload_state(case.h0, case.g0)
        e.run(20)
        files.write_fields(e, p, float32=f32, deflate=deflate)
        f = e.download()
    finally:
        e.free()
    for name, key in (("density", "rho"), ("concentration", "c"), ("u_x", "ux"), ("u_y", "uy"), ("u_z", "uz"),
                      ("pressure", "p")):
        got = files.read_dataset(p, name)
        assert got.dtype == (np.float32 if f32 else np.float64)
        assert np.array_equal(got, f[key].astype(got.dtype)), name
