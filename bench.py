#!/usr/bin/env python
"""Benchmark of the Lee–Liu D3Q19 step on B200: MLUPS and HBM-roofline fraction.

Workload (the production dispersion configuration at 300^3): a seeded Gaussian
random field (correlation length 6 lu) thresholded at porosity 0.37, largest
x-percolating cluster kept (~10M fluid sites), periodic, body force 1e-6 along
x, fused MRT, contact angle 45 deg, correct_op_mass on, slab initial condition,
FP32 population storage. A step is one pass of the hot path over the whole
lattice (the driver loop body: step + mass correction). Synthetic data: the
reference's TIFF image stacks are not available, the random field stands in
with the same size and porosity.

Arms:
  default          this engine (hand-written sm_100a kernels via the C-ABI)
  --impl reference the reference's CPU path on this box's host cores: the CPU
                   oracle (C++/OpenMP restatement of the reference step; the
                   reference's own CPU engine lives in the absent felbm_local
                   tree), on a bounded sample of the same workload per step.

Multi-GPU (torchrun, N ranks): independent replicas, one lattice per GPU, no
collective on the data path ("scaling": "weak"); the timed region is
bracketed by barriers and the max over ranks is reported.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

Q = 19
B_ALG = {"f64": 904, "f32": 452, "f16s": 262, "bf16s": 262}       # bytes / site / step (whole step)
B_P4 = {"f64": 8 * (19 + 4 + 38), "f32": 4 * (19 + 4 + 38), "f16s": 2 * 19 + 4 * 4 + 2 * 38,
        "bf16s": 2 * 19 + 4 * 4 + 2 * 38}                          # collide pass: g, 4 fields in; h, g out
METRIC = "MLUPS (fluid-site lattice updates / s, 1e6) at 300^3 porous, fused MRT"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=300)
    ap.add_argument("--storage", default="f32", choices=["f64", "f32", "f16s", "bf16s"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    lrank = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, lrank


def workload(size: int, seed: int = 2024):
    """The production dispersion configuration: fluid physics of the
    reference's cfg/3d_image/params.cfg (rho0 = rho1 = 1, tau = 0.9, W = 5,
    sigma = 0.0083, mobility_coeff 0.02) with a 45 degree contact angle
    (phi = 6 sigma cos 45) and body force 1e-6 along x."""
    from felbm_gpu_b200 import default_params, geometry
    shape = (size, size, size)
    solid, por = geometry.grf(shape, 6.0, 0.37, seed, flow_axis=0)
    sigma, W = 0.0083, 5.0
    p = default_params(rho0=1.0, rho1=1.0, tau0=0.9, tau1=0.9, surface_tension=sigma, interface_width=W,
                       mobility_coeff=0.02, phi=6 * sigma * np.cos(np.radians(45.0)), gx=1e-6,
                       use_mrt=1, use_halfway_bb=1, correct_op_mass=1,
                       stream_matrix_free=1, grad_matrix_free=1, fused=1, fuse_collision=1,
                       mrt_fast_transform=1, stream_inplace=1)
    c = geometry.order_parameter(solid, "slab", W, origin=(0, 0, 0), axis=0, thickness=size // 2)
    h, g = geometry.equilibrium(c, 1.0, p.rho0, p.rho1)
    return solid, por, p, h, g


class Clocks:
    """nvidia-smi sampler for the timed region (SM clock, reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(storage: str, size: int):
    """Per-launch DRAM bytes of the collide kernel from the committed ncu
    summary (profiles/collide_traffic.json), scaled to this lattice."""
    path = os.path.join(ROOT, "profiles", "collide_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        rec = d.get(storage)
        if rec:
            return rec["bytes_per_site"]
    except Exception:
        pass
    return None


def cpu_sample_mlups(storage_label: str, seconds: float = 12.0):
    """The CPU oracle on a bounded sample of the workload: a 100^3 lattice of
    the same random-field construction, all host threads, steps until ~seconds."""
    from oracle.oracle_py import Oracle
    solid, por, p, h, g = workload(100, seed=99)
    o = Oracle(p, solid)
    o.upload_state(h, g)
    o.record_target_mass()
    o.run(1, 0)
    steps, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        o.run(1, steps + 1)
        steps += 1
    dt = time.perf_counter() - t0
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": o.n * steps / dt / 1e6, "unit": "MLUPS", "cores": cores, "kind": "port",
            "sample": f"CPU oracle (FP64, OpenMP) on a 100^3 GRF sample of the same construction "
                      f"({o.n} sites), {steps} steps in {dt:.1f} s"}


def run_reference_arm(args, ws, rank):
    if rank != 0:
        return 0
    from oracle.oracle_py import Oracle
    solid, por, p, h, g = workload(100, seed=99)
    o = Oracle(p, solid)
    o.upload_state(h, g)
    o.record_target_mass()
    o.run(max(args.warmup, 1), 0)
    t0 = time.perf_counter()
    o.run(args.steps, args.warmup)
    dt = time.perf_counter() - t0
    v = o.n * args.steps / dt / 1e6
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    line = {"metric": METRIC, "value": v, "unit": "MLUPS", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": "GRF porous sample 100^3 (same construction as the 300^3 workload), "
                                   "fused MRT, correct_op_mass", "sites": int(o.n)},
            "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": cores, "kind": "port",
                             "sample": f"CPU oracle (C++/OpenMP restatement of the reference step) on a 100^3 "
                                       f"sample ({o.n} sites) per step; the reference's own CPU engine "
                                       f"(felbm_local) is not in the reference snapshot"},
            "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    ws, rank, lrank = dist_env()
    if args.impl == "reference":
        return run_reference_arm(args, ws, rank)
    import torch
    torch.cuda.set_device(lrank)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from felbm_gpu_b200 import MultiPhaseGPU
    from felbm_gpu_b200 import _capi
    solid, por, p, h0, g0 = workload(args.size, seed=2024 + rank)
    p.storage = _capi.STORAGE[args.storage]
    eng = MultiPhaseGPU(p, solid, device=lrank)
    n = eng.n
    eng.upload_state(h0, g0)
    eng.record_target_mass()
    eng.run(max(args.warmup, 3))
    torch.cuda.synchronize()

    def barrier():
        if dist:
            dist.barrier()

    l0 = eng.launch_count()
    with Clocks(lrank) as clk:
        barrier()
        torch.cuda.synchronize()
        ms = eng.time_run(args.steps)
        torch.cuda.synchronize()
        barrier()
    launches = eng.launch_count() - l0
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        nt = torch.tensor([float(n)], device="cuda")
        dist.all_reduce(nt)
        n_total = nt.item()
    else:
        n_total = n
    value = n_total * args.steps / (ms / 1e3) / 1e6
    # per-kernel device times (plain launches, CUDA events on the engine stream)
    kms = eng.time_kernels(max(10, min(args.steps, 50))) / max(10, min(args.steps, 50))
    peak, peak_kind = measured_peak()
    t_p4 = kms[4] / 1e3
    achieved = B_P4[args.storage] * n / t_p4 / 1e9
    tr = profiled_traffic(args.storage, args.size)
    roof = {"bound": "hbm", "kernel": "k_collide (P4: equilibria + Guo force + MRT, push streaming)",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_kind": peak_kind,
            "algorithmic_bytes_per_site": B_P4[args.storage],
            "traffic": (tr * n if tr else None),
            "step_achieved": B_ALG[args.storage] * n * args.steps / (ms / 1e3) / 1e9,
            "step_frac": B_ALG[args.storage] * n * args.steps / (ms / 1e3) / 1e9 / peak,
            "step_algorithmic_bytes_per_site": B_ALG[args.storage],
            "kernel_ms": {"moments": kms[0], "open_bnd": kms[1], "cfield": kms[2], "lapmu": kms[3],
                          "collide": kms[4]}}
    e2e = None
    if not args.no_e2e:
        # One job through the public API with host buffers: the initial state
        # goes host->device (fe_upload_state, FP64 in the reference layout),
        # then the reference driver loop runs K steps (per step the forcing
        # factor goes host->device, step + mass correction, and the flow
        # statistics come back device->host), and the final state comes back
        # (fe_download_state). Host wall clock around all of it.
        ke = args.steps
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        eng.upload_state(h0, g0)
        eng.record_target_mass()
        for _ in range(ke):
            eng.set_forcing_factor(1.0)
            eng.step(1)
            eng.apply_mass_correction(want_drift=False)
            eng.flow_stats()
        hd, gd = eng.download_state()
        torch.cuda.synchronize()
        barrier()
        dt = time.perf_counter() - t0
        del hd, gd
        if dist:
            tt = torch.tensor([dt], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            dt = float(tt.item())
        state_bytes = h0.nbytes + g0.nbytes
        e2e = {"value": n_total * ke / dt / 1e6, "unit": "MLUPS",
               "h2d_bytes_per_step": (state_bytes + ke * 8) / ke,
               "d2h_bytes_per_step": (state_bytes + ke * 48 + 16) / ke, "steps": ke,
               "what": "one job: fe_upload_state (host FP64 state) + K x (fe_set_forcing_factor, fe_step, "
                       "fe_apply_mass_correction, fe_flow_stats) + fe_download_state, host wall clock"}
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_sample_mlups(args.storage)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": args.storage, "data": "synthetic",
                "config": {"workload": f"{args.size}^3 GRF porous (corr 6, porosity 0.37, largest cluster), "
                                       f"periodic, body force 1e-6, fused MRT, theta 45, correct_op_mass, "
                                       f"slab IC, {args.storage} populations",
                           "sites": int(n), "porosity": por, "parallelism": f"replicas x{ws}",
                           "l2": "inputs larger than L2 (state > 1 GB), no flush"},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    eng.free()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
