"""Helpers of the drop-in tests: a settings.cfg / params.cfg pair in the
reference driver's format (cfg/*/settings.cfg keys), the case files the C++
driver (tests/cpp/drop_in_driver.cpp) reads, and its build with g++ against
include/felbm_b200.hpp and the library."""
from __future__ import annotations

import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER_SRC = os.path.join(ROOT, "tests", "cpp", "drop_in_driver.cpp")
LIB_DIR = os.path.join(ROOT, "felbm_gpu_b200", "_lib")

SETTINGS = """\
# settings of a drop-in test run (the reference driver's key names)
model           = multi_phase
logging         = true
console         = false
output_dir      = ./out/
output_name     = output
timeseries_file = series.txt
output_float32  = true        # [gpu] float32 fields
output_deflate  = {deflate}           # [gpu] gzip level
log_skip        = {log_skip}
file_skip       = 1000
size_x          = {nx}
size_y          = {ny}
size_z          = {nz}
velocity_set    = d3q19
threads         = 32
num_subdomains  = 1
use_halfway_bb  = true
domain_geometry = spheres_repulsive
param_file      = params.cfg
max_iterations  = {steps}
acceleration_x  = 1.0e-05
acceleration_y  = 0.0
acceleration_z  = 0.0
forcing_x       = 2.0e-04
forcing_y       = -1.0e-04
forcing_z       = 0.0
forcing_timedep = "sinusoidal"
forcing_period  = 30.0
use_open_bnd    = false
in_out_dir      = 0
use_inlet_pressure  = false
pressure_inlet      = 0.0
fluid_initializer   = droplet
use_mrt             = true
mrt_lambda          = 0.1875
correct_op_mass     = true
particles_enable    = false
stream_matrix_free = true
grad_matrix_free   = true
fused              = true
fuse_collision     = true
mrt_fast_transform = true     # [gpu]
stream_inplace     = true     # [gpu]
checkpoint_skip    = 500      # [gpu]
gpu_device         = {device}
"""

PARAMS = """\
rho0            = 5.0
rho1            = 1.0
tau0            = 1.0
tau1            = 1.0
density_solid   = 20.0
interface_width = 4.0
surface_tension = 0.01
mobility_coeff  = 0.02
phi             = 0.03
"""


def write_cfg(d: str, shape, steps: int = 60, log_skip: int = 10, deflate: int = 0, device: int = -1) -> str:
    nz, ny, nx = shape
    with open(os.path.join(d, "settings.cfg"), "w") as f:
        f.write(SETTINGS.format(nx=nx, ny=ny, nz=nz, steps=steps, log_skip=log_skip, deflate=deflate,
                                device=device))
    with open(os.path.join(d, "params.cfg"), "w") as f:
        f.write(PARAMS)
    return os.path.join(d, "settings.cfg")


def write_case(d: str, solid: np.ndarray, h0: np.ndarray, g0: np.ndarray):
    np.ascontiguousarray(solid, np.uint8).tofile(os.path.join(d, "solid.bin"))
    np.ascontiguousarray(h0, np.float64).tofile(os.path.join(d, "h0.bin"))
    np.ascontiguousarray(g0, np.float64).tofile(os.path.join(d, "g0.bin"))


def build_driver(out_dir: str) -> str:
    exe = os.path.join(out_dir, "drop_in_driver")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), DRIVER_SRC, "-o", exe,
                    "-L", LIB_DIR, "-lfelbm_b200", f"-Wl,-rpath,{LIB_DIR}"], check=True)
    return exe
