"""The reference driver's configuration files through fe_cfg_read, and the
C++ drop-in: a driver written against include/felbm_b200.hpp compiles and
links against the library (its run is a GPU test)."""
import os
import subprocess

import pytest

from drop_in import build_driver, write_cfg
from felbm_gpu_b200 import default_params
from felbm_gpu_b200.engine import read_cfg


def test_settings_and_params_keys(tmp_path):
    path = write_cfg(str(tmp_path), (8, 12, 16), steps=60, log_skip=10, deflate=4)
    p, ob, d, log = read_cfg(path)
    # params.cfg
    assert (p.rho0, p.rho1, p.tau0, p.tau1) == (5.0, 1.0, 1.0, 1.0)
    assert (p.interface_width, p.surface_tension, p.mobility_coeff, p.phi) == (4.0, 0.01, 0.02, 0.03)
    # derived as fe_params_derive does (compare_cpu_gpu.cu:115-118)
    assert abs(p.kappa - 1.5 * 4.0 * 0.01) < 1e-15 and abs(p.beta - 12 * 0.01 / 4.0) < 1e-15
    # settings.cfg solver keys
    assert (p.gx, p.fx, p.fy) == (1e-5, 2e-4, -1e-4)
    assert p.forcing_timedep == 1 and p.forcing_period == 30.0
    assert p.use_mrt == 1 and p.mrt_lambda == 0.1875 and p.use_halfway_bb == 1 and p.correct_op_mass == 1
    for k in ("stream_matrix_free", "grad_matrix_free", "fused", "fuse_collision", "mrt_fast_transform",
              "stream_inplace"):
        assert getattr(p, k) == 1, k
    # driver-level keys
    assert (d["size_x"], d["size_y"], d["size_z"]) == (16, 12, 8)
    assert d["max_iterations"] == 60 and d["log_skip"] == 10 and d["checkpoint_skip"] == 500
    assert d["output_deflate"] == 4 and d["output_float32"] == 1 and d["gpu_device"] == -1
    assert d["output_name"] == "output" and d["param_file"] == "params.cfg"
    assert d["domain_geometry"] == "spheres_repulsive" and d["restart_file"] == ""
    assert d["unknown_keys"] >= 2  # threads, num_subdomains, density_solid ...
    # every switch is logged with the path it selects
    lines = log.strip().splitlines()
    assert len(lines) == 6 and all("->" in ln for ln in lines)


def test_open_boundary_keys(tmp_path):
    path = write_cfg(str(tmp_path), (8, 8, 8))
    txt = open(path).read().replace("correct_op_mass     = true", "correct_op_mass     = false")
    txt += ("use_open_bnd = true\nuse_inlet_pressure = true\npressure_inlet = 1.005\nuse_outlet_pressure = true\n"
            "pressure_outlet = 1.0\nuse_inlet_fluid = true\ninlet_fluid = 1\noutlet_fluid = 0\n"
            "inlet_mode = \"stripes\"\ninlet_split_dir = \"z\"\ninlet_period = 8\ninlet_duty = 0.25\n"
            "inlet_ramp = 2\ninlet_split_pos = 3\ncopy_to_buffers = true\n")
    open(path, "w").write(txt)
    p, ob, d, _ = read_cfg(path)
    assert d["use_open_bnd"] == 1
    assert ob.use_in_prs and ob.p_in == 1.005 and ob.use_out_prs and ob.p_out == 1.0 and ob.use_in_fluid
    # felbm_gpu_main.cu:352-355: c_out_fixed = 1 - outlet_fluid, inlet_c_a = 1 - inlet_fluid
    assert ob.inlet_c_a == 0.0 and ob.c_out_fixed == 1.0 and ob.rho_out_fixed == p.rho0
    assert ob.inlet_mode == 3 and ob.split_axis == 2 and ob.inlet_period == 8 and ob.inlet_duty == 0.25
    assert ob.inlet_ramp == 2 and ob.split_pos == 3 and ob.copy_to_buffers


def test_refusals_and_errors(tmp_path):
    path = write_cfg(str(tmp_path), (8, 8, 8))
    base = open(path).read()
    # the reference driver refuses mass correction with open boundaries
    open(path, "w").write(base + "use_open_bnd = true\n")
    with pytest.raises(Exception, match="correct_op_mass"):
        read_cfg(path)
    open(path, "w").write(base.replace("multi_phase", "single_phase"))
    with pytest.raises(Exception, match="single_phase"):
        read_cfg(path)
    open(path, "w").write(base.replace("log_skip        = 10", "log_skip = ten"))
    with pytest.raises(Exception, match="log_skip"):
        read_cfg(path)
    with pytest.raises(Exception, match="cannot open"):
        read_cfg(str(tmp_path / "missing.cfg"))


def test_keys_absent_keep_the_given_values(tmp_path):
    (tmp_path / "settings.cfg").write_text("model = multi_phase\nparam_file = params.cfg\n")
    (tmp_path / "params.cfg").write_text("rho0 = 2.0\n")
    base = default_params(tau0=0.7, gx=3e-6, use_mrt=1)
    p, _, d, _ = read_cfg(str(tmp_path / "settings.cfg"), base)
    assert p.rho0 == 2.0 and p.tau0 == 0.7 and p.gx == 3e-6 and p.use_mrt == 1


def test_cpp_driver_builds_and_reports_no_device(tmp_path):
    """The drop-in driver compiles against include/felbm_b200.hpp and links
    against the library; without a GPU it stops with the engine's
    no-device status (FE_ERR_NO_DEVICE = 3, exit code 13), no exit() inside."""
    exe = build_driver(str(tmp_path))
    import numpy as np
    from drop_in import write_case
    path = write_cfg(str(tmp_path), (4, 4, 4), steps=2)
    write_case(str(tmp_path), np.zeros((4, 4, 4), np.uint8), np.zeros(19 * 64), np.zeros(19 * 64))
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present: the driver's run is tests/test_gpu_drop_in.py")
    r = subprocess.run([exe, path, str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 13, (r.returncode, r.stderr)
    assert "no CUDA device" in r.stderr
    assert os.path.exists(tmp_path / "switches.txt")
