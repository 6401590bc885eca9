#!/usr/bin/env python
"""Generate the golden vectors of tests/golden/*.npz.

Each file holds the state and fields after 20 steps (the reference's
validation step count, scripts/validate.sh:37-50) of one parity case from
tests/cases.py, computed by the reference's OWN kernels: matNBI/felbm_gpu's
include/felbm_gpu/device_engine.cuh compiled unmodified for sm_100a (FP64) by
oracle/ref/build_ref.sh and driven in MultiPhaseGPU::step order
(oracle/ref/ref_harness.cu). Needs a GPU. To keep the files small, a seeded
subset of the 19n state entries and of the sites is stored, plus the state
sums.

    python tests/golden/make_golden.py <outdir>
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from cases import make_case  # noqa: E402
from oracle import ref_py  # noqa: E402
from oracle.oracle_py import Oracle  # noqa: E402

STEPS = 20
SPECS = [
    ("fluid_bgk", {}), ("spheres_bgk", {}), ("spheres_mrt", {}), ("spheres_mrt_wet", {}),
    ("cyl2d_mrt", {"ref_rates": True}), ("grf_mrt_mass", {}), ("grf_bgk_mass", {}),
    ("openbnd_bgk", {}), ("openbnd_bgk", {"inlet_mode": 1}), ("openbnd_bgk", {"inlet_mode": 2}),
    ("openbnd_mrt_buf", {}), ("openbnd_mrt_buf", {"inlet_mode": 4}),
]


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    rng = np.random.default_rng(1234)
    for name, kw in SPECS:
        case = make_case(name, **dict(kw))
        o = Oracle(case.params, case.solid)
        r = ref_py.RefKernels(case.params, o, precision="f64")
        if case.open_bnd is not None:
            r.set_open_bnd(case.open_bnd)
        r.upload_state(case.h0, case.g0)
        if case.correct_mass:
            r.record_target_mass()
        for _ in range(STEPS):
            r.step(1)
            r.apply_mass_correction()
        h, g = r.download_state()
        f = r.fields()
        r.close()
        sel = np.sort(rng.choice(len(h), size=min(1500, len(h)), replace=False))
        sites = np.sort(rng.choice(o.n, size=min(400, o.n), replace=False))
        tag = name + "".join(f"_{k}{v}" for k, v in kw.items())
        out = dict(case=name, steps=STEPS, sel=sel, h=h[sel], g=g[sel], h_sum=h.sum(), g_sum=g.sum(),
                   sites=sites)
        for k, v in kw.items():
            out["kw_" + k] = np.array(v)
        for k, v in f.items():
            out["f_" + k] = v[sites]
        np.savez_compressed(os.path.join(outdir, f"ref_{tag}.npz"), **out)
        print("wrote", tag, "n =", o.n)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
