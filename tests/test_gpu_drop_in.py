"""The C++ drop-in on the GPU: tests/cpp/drop_in_driver.cpp, built with g++
against include/felbm_b200.hpp, reads settings.cfg + params.cfg, runs the
reference driver's loop (forcing factor of step t, step, mass correction,
asynchronous statistics every log_skip steps) and writes its final state;
the CPU oracle runs the same loop on the same parameters (read by the same
cfg reader) and initial state: FP64 storage, within 1e-12."""
import math
import subprocess

import numpy as np
import pytest

from cases import make_case
from drop_in import build_driver, write_case, write_cfg
from felbm_gpu_b200.engine import read_cfg
from oracle.oracle_py import Oracle

pytestmark = pytest.mark.gpu


def test_cpp_driver_matches_oracle(require_gpu, tmp_path):
    case = make_case("spheres_mrt_wet")
    steps = 60
    path = write_cfg(str(tmp_path), case.solid.shape, steps=steps, log_skip=10)
    write_case(str(tmp_path), case.solid, case.h0, case.g0)
    exe = build_driver(str(tmp_path))
    r = subprocess.run([exe, path, str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    h = np.fromfile(tmp_path / "h.bin")
    g = np.fromfile(tmp_path / "g.bin")
    p, _, d, log = read_cfg(path)
    assert open(tmp_path / "switches.txt").read() == log
    o = Oracle(p, case.solid)
    o.upload_state(case.h0, case.g0)
    o.record_target_mass()
    for t in range(steps):
        o.set_forcing_factor(math.sin(2.0 * math.pi * t / p.forcing_period))
        o.step(1)
        o.apply_mass_correction()
    ho, go = o.download_state()
    assert np.max(np.abs(h - ho)) <= 1e-12, np.max(np.abs(h - ho))
    assert np.max(np.abs(g - go)) <= 1e-12, np.max(np.abs(g - go))
    # statistics every log_skip steps, collected asynchronously
    rows = np.loadtxt(tmp_path / "series.txt")
    assert rows.shape == (steps // 10, 7) and list(rows[:, 0]) == list(range(10, steps + 1, 10))
    assert np.allclose(rows[-1, 1:], o.flow_stats(), rtol=1e-10, atol=1e-14)
