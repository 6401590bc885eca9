#!/usr/bin/env python
"""Times the reference's own device kernels on a B200 — comparator only.

The kernels are matNBI/felbm_gpu's include/felbm_gpu/device_engine.cuh,
compiled unmodified for sm_100a by oracle/ref/build_ref.sh and driven in the
MultiPhaseGPU::step order (multiphase_gpu.cuh:522-631: moments, gradients,
Laplacians, fused collision, gather streaming) by oracle/ref/ref_harness.cu,
on the neighbour/case tables of the CPU oracle. The workload is the bench's
production configuration (random-field porous medium, fused MRT, mass
correction) at a size whose tables fit host memory. Prints one JSON line:
step-only throughput and the reference driver loop (step + mass correction,
felbm_gpu_main.cu:741-748), in fluid-site updates per second.

    python oracle/ref/bench_ref_kernels.py --size 200 --steps 50 --precision f32
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=200)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"])
    args = ap.parse_args()

    from bench import workload
    from oracle.oracle_py import Oracle
    from oracle.ref_py import RefKernels, available

    if not available(args.precision):
        print(json.dumps({"impl": "reference kernels", "unavailable": "oracle/_ref not built"}))
        return 0
    solid, por, p, h, g = workload(args.size)
    o = Oracle(p, solid)
    r = RefKernels(p, o, precision=args.precision)
    n = r.n
    del o
    r.upload_state(h, g)
    r.record_target_mass()
    lib, hd = r.lib, r._h
    for _ in range(args.warmup):
        lib.ref_step(hd)
        r.apply_mass_correction()
    assert lib.ref_sync() == 0
    # the reference driver loop: step + mass correction (a host readback)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        lib.ref_step(hd)
        r.apply_mass_correction()
    assert lib.ref_sync() == 0
    dt_loop = time.perf_counter() - t0
    # steps alone (queued back to back)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        lib.ref_step(hd)
    assert lib.ref_sync() == 0
    dt_step = time.perf_counter() - t0
    r.close()
    print(json.dumps({
        "impl": "reference device_engine.cuh kernels, unmodified, sm_100a",
        "precision": args.precision, "workload": f"{args.size}^3 GRF porous (corr 6, porosity 0.37), fused MRT, "
                                                 f"correct_op_mass, slab IC", "sites": n, "porosity": por,
        "steps": args.steps,
        "mlups_step_plus_correction": n * args.steps / dt_loop / 1e6,
        "ms_per_step_plus_correction": dt_loop * 1e3 / args.steps,
        "mlups_step": n * args.steps / dt_step / 1e6,
        "ms_per_step": dt_step * 1e3 / args.steps,
        "clock": "host wall clock around queued steps, device synchronised on both sides",
    }), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
