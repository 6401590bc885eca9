"""Reduced-precision storages against the FP64 oracle: populations stored in
FP32, or as scaled FP16 / BF16 deviations from the rest state (g only:
f16g, bf16g; h and g: f16s, bf16s), arithmetic in FP32 registers.

Each storage's error after 200 steps is bounded by a stated value (about
twice the measured one, so the bound catches a regression, not rounding
noise): max|dc|, max|du| (vector magnitude) and, for the mass-corrected
case, the relative order-parameter mass drift of the downloaded state; for
the uncorrected cylinder pack, the drift's difference from the oracle's own.
"""
import numpy as np
import pytest

from cases import make_case
from parity import run_engine, run_oracle

pytestmark = pytest.mark.gpu

STEPS = 200
# (case, storage): (max|dc|, max|du|, mass bound)
BOUNDS = {
    ("grf_mrt_mass", "f32"): (2e-5, 5e-7, 1e-8),
    ("grf_mrt_mass", "f16g"): (5e-5, 2e-6, 1e-8),
    ("grf_mrt_mass", "bf16g"): (5e-4, 2e-5, 1e-8),
    ("grf_mrt_mass", "f16s"): (2e-3, 2e-6, 6e-5),
    ("grf_mrt_mass", "bf16s"): (0.1, 1e-4, 4e-4),
    ("cyl2d_mrt", "f32"): (3e-5, 2e-6, 1e-6),
    ("cyl2d_mrt", "f16g"): (3e-5, 2e-6, 1e-6),
    ("cyl2d_mrt", "bf16g"): (3e-5, 3e-6, 1e-6),
    ("cyl2d_mrt", "f16s"): (1.2e-2, 2e-6, 3e-3),
    ("cyl2d_mrt", "bf16s"): (8e-2, 5e-5, 1.2e-2),
}

_oracle_cache = {}


def oracle_result(name):
    if name not in _oracle_cache:
        _oracle_cache[name] = run_oracle(make_case(name), STEPS)
    return _oracle_cache[name]


@pytest.mark.parametrize("name,storage", sorted(BOUNDS))
def test_storage_error_vs_fp64_oracle(require_gpu, name, storage):
    case = make_case(name)
    h, g, f, _, _ = run_engine(case, STEPS, storage)
    ho, go, fo, _ = oracle_result(name)
    dc = float(np.max(np.abs(f["c"] - fo["c"])))
    du = float(np.max(np.sqrt((f["ux"] - fo["ux"]) ** 2 + (f["uy"] - fo["uy"]) ** 2 + (f["uz"] - fo["uz"]) ** 2)))
    m0 = float(np.sum(case.h0))
    drift = abs(float(np.sum(h)) - m0) / abs(m0)
    drift_oracle = abs(float(np.sum(ho)) - m0) / abs(m0)
    bc, bu, bm = BOUNDS[(name, storage)]
    print(f"{name} {storage}: max|dc| {dc:.2e} max|du| {du:.2e} drift {drift:.2e} (oracle {drift_oracle:.2e})")
    assert dc <= bc, dc
    assert du <= bu, du
    if case.correct_mass:
        assert drift <= bm, drift
    else:
        assert abs(drift - drift_oracle) <= bm, (drift, drift_oracle)
