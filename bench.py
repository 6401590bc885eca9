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
B_ALG = {"f64": 904, "f32": 452, "f16s": 262, "bf16s": 262,       # bytes / site / step (whole step)
         "f16g": 338, "bf16g": 338}                                # h FP32 (38 moves), g 16-bit (57 moves)
B_P4 = {"f64": 8 * (19 + 4 + 38), "f32": 4 * (19 + 4 + 38), "f16s": 2 * 19 + 4 * 4 + 2 * 38,
        "bf16s": 2 * 19 + 4 * 4 + 2 * 38,                          # collide pass: g, 4 fields in; h, g out
        "f16g": 2 * 19 + 4 * 4 + 4 * 19 + 2 * 19, "bf16g": 2 * 19 + 4 * 4 + 4 * 19 + 2 * 19}
METRIC = "MLUPS (fluid-site lattice updates / s, 1e6) at 300^3 porous, fused MRT"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=300)
    ap.add_argument("--storage", default="f32", choices=["f64", "f32", "f16s", "bf16s", "f16g", "bf16g"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the served sweep and request stream")
    ap.add_argument("--no-tracers", action="store_true", help="skip the production loop with 12,000 tracers")
    ap.add_argument("--no-autotune", action="store_true",
                    help="skip the layout autotuner (default bricks, two steps per graph launch)")
    ap.add_argument("--brick", default="auto", choices=["auto", "8x8x8", "8x8x4", "16x8x8"],
                    help="force a brick shape (skips the autotuner)")
    ap.add_argument("--sweep-steps", type=int, default=1000, help="steps per solve of the 64-solve sweep")
    ap.add_argument("--stream-seconds", type=float, default=15.0, help="arrival window of the request stream")
    ap.add_argument("--stream-rate", type=float, default=4.0, help="Poisson arrival rate (requests / s)")
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


def profiled_traffic(storage: str, size: int, brick: str = "8x8x8"):
    """Per-site DRAM bytes of the collide kernel with this brick from the
    committed ncu summary (profiles/collide_traffic.json), to be scaled to
    this lattice; None when that layout was not captured."""
    path = os.path.join(ROOT, "profiles", "collide_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        rec = (d.get(storage) or {}).get(brick)
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


def sweep_specs(count: int, steps: int, seed: int = 7):
    """The batching sweep: uneven solves, 2-D cylinder packs 64^2 to 512^2 and
    3-D random-field media 48^3 to 128^3, porosity U[0.3, 0.6], contact angle
    U[30, 150] deg, mobility coefficient U[0.005, 0.05], MRT, mass correction,
    slab initial condition, body force 1e-6."""
    from felbm_gpu_b200 import default_params, geometry
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        por, theta, mob = rng.uniform(0.3, 0.6), rng.uniform(30, 150), rng.uniform(0.005, 0.05)
        if k % 2 == 0:
            L = int(rng.integers(64, 513))
            solid, _ = geometry.cylinders((1, L, L), 6.0, 12.0, por, seed=seed * 1000 + k)
        else:
            L = int(rng.integers(48, 129))
            solid, _ = geometry.grf((L, L, L), 6.0, por, seed=seed * 1000 + k, flow_axis=0)
        sigma, W = 1e-3, 4.0
        p = default_params(rho0=1.0, rho1=1.0, tau0=1.0, tau1=1.0, surface_tension=sigma, interface_width=W,
                           mobility_coeff=mob, phi=6 * sigma * np.cos(np.radians(theta)), gx=1e-6, use_mrt=1,
                           correct_op_mass=1)
        out.append({"params": p, "solid": solid, "init": (1, (0.0, 0.0, 0.0, 0.0, L / 2)), "W": W,
                    "steps": steps, "sites": int(np.count_nonzero(solid == 0))})
    return out


def stream_specs(seconds: float, rate: float, seed: int = 11):
    """The served request stream: Poisson arrivals; geometry (2-D pack or 3-D
    random field), size log-uniform 64^2 x 1 .. 200^3, contact angle and step
    count drawn from the seed. Step counts are 1/20 of the workload's
    1000-20,000 (50-1000) so the stream fits a short run."""
    from felbm_gpu_b200 import default_params, geometry
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > seconds:
            break
        k = len(out)
        sites_target = float(np.exp(rng.uniform(np.log(64 ** 2), np.log(200 ** 3))))
        por, theta = rng.uniform(0.3, 0.6), rng.uniform(30, 150)
        if sites_target < 512 ** 2 and rng.random() < 0.5:
            L = max(64, int(round(np.sqrt(sites_target))))
            solid, _ = geometry.cylinders((1, L, L), 6.0, 12.0, por, seed=seed * 1000 + k)
        else:
            L = int(np.clip(round(sites_target ** (1 / 3)), 48, 200))
            solid, _ = geometry.grf((L, L, L), 6.0, por, seed=seed * 1000 + k, flow_axis=0)
        sigma, W = 1e-3, 4.0
        p = default_params(rho0=1.0, rho1=1.0, tau0=1.0, tau1=1.0, surface_tension=sigma, interface_width=W,
                           mobility_coeff=0.02, phi=6 * sigma * np.cos(np.radians(theta)), gx=1e-6, use_mrt=1,
                           correct_op_mass=1)
        out.append({"arrival": t, "params": p, "solid": solid, "init": (1, (0.0, 0.0, 0.0, 0.0, L / 2)),
                    "W": W, "steps": int(rng.integers(50, 1001)), "sites": int(np.count_nonzero(solid == 0))})
    return out


def run_alone(spec, storage: str):
    """One solve through the plain engine: create, upload, run, fields back."""
    from felbm_gpu_b200 import MultiPhaseGPU, _capi, geometry
    import ctypes as C
    p = _capi.FeParams()
    C.pointer(p)[0] = spec["params"]
    p.storage = _capi.STORAGE[storage]
    kind, a = spec["init"]
    c = geometry.order_parameter(spec["solid"], "slab", spec["W"], origin=a[:3], axis=int(a[3]), thickness=a[4])
    h0, g0 = geometry.equilibrium(c, 1.0, p.rho0, p.rho1)
    e = MultiPhaseGPU(p, spec["solid"])
    try:
        e.upload_state(h0, g0)
        e.record_target_mass()
        e.run(spec["steps"])
        return e.download(), e.current_mass(), e.get_target_mass()
    finally:
        e.free()


def serve_legs(args):
    """Served sweep and request stream against the plain engine on the same GPU."""
    import torch
    from felbm_gpu_b200.serving import Server
    storage = "f32"
    out = {}
    # -- the 64-solve sweep: all submitted at once --------------------------
    specs = sweep_specs(64, args.sweep_steps)
    work = sum(s["sites"] * s["steps"] for s in specs)
    run_alone(specs[0], storage)  # warm-up (library, context, kernels)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    seq = [run_alone(s, storage) for s in specs]
    t_seq = time.perf_counter() - t0
    srv = Server(storage=storage, chunk_steps=50)
    t0 = time.perf_counter()
    for k, s in enumerate(specs):
        srv.submit(k, s["params"], s["solid"], s["steps"], init=s["init"], init_width=s["W"])
    res = []
    while len(res) < len(specs):
        res += srv.poll()
        time.sleep(0.002)
    t_srv = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    res.sort(key=lambda r: r.id)
    same = all(r.status == 0 and np.array_equal(r.fields["c"], seq[r.id][0]["c"]) for r in res)
    dc = max(float(np.max(np.abs(r.fields["c"] - seq[r.id][0]["c"]))) for r in res)
    drift = max(abs(r.mass_final - r.mass0) / abs(r.mass0) for r in res)
    out["sweep"] = {"solves": len(specs), "steps_each": args.sweep_steps, "site_updates": work,
                    "served_mlups": work / t_srv / 1e6, "sequential_mlups": work / t_seq / 1e6,
                    "speedup": t_seq / t_srv, "served_s": t_srv, "sequential_s": t_seq,
                    "ttr_p50_s": st["ttr_p50"], "ttr_p99_s": st["ttr_p99"],
                    "results_identical_to_alone": bool(same), "max_abs_dc_vs_alone": dc,
                    "max_rel_mass_drift": drift,
                    "what": "64 uneven solves (2-D packs 64^2-512^2, 3-D GRF 48^3-128^3, porosity, angle, "
                            "mobility from seed 7), MRT FP32, submitted together to the request loop vs run one "
                            "after another through the plain engine; both include engine creation, upload and "
                            "field download; host wall clock"}
    # -- the Poisson request stream -----------------------------------------
    reqs = stream_specs(args.stream_seconds, args.stream_rate)
    if reqs:
        srv = Server(storage=storage, chunk_steps=50)
        t0 = time.perf_counter()
        res, nxt = [], 0
        while len(res) < len(reqs):
            now = time.perf_counter() - t0
            while nxt < len(reqs) and reqs[nxt]["arrival"] <= now:
                s = reqs[nxt]
                srv.submit(nxt, s["params"], s["solid"], s["steps"], init=s["init"], init_width=s["W"],
                           want_fields=False)
                nxt += 1
            res += srv.poll()
            time.sleep(0.002)
        t_srv = time.perf_counter() - t0
        st = srv.stats()
        srv.close()
        ttr = np.array([r.time_to_result for r in res])
        # the same requests, one after another through the plain engine: a
        # request starts at its arrival or when the previous one finished
        durs = []
        for s in reqs:
            t1 = time.perf_counter()
            run_alone(s, storage)
            durs.append(time.perf_counter() - t1)
        free_at, ttr_seq = 0.0, []
        for s, d in zip(reqs, durs):
            start = max(s["arrival"], free_at)
            free_at = start + d
            ttr_seq.append(free_at - s["arrival"])
        work = sum(s["sites"] * s["steps"] for s in reqs)
        out["stream"] = {"requests": len(reqs), "rate_per_s": args.stream_rate, "window_s": args.stream_seconds,
                         "site_updates": work, "served_mlups_busy": st["mlups_busy"],
                         "served_ttr_p50_s": float(np.percentile(ttr, 50)),
                         "served_ttr_p99_s": float(np.percentile(ttr, 99)),
                         "sequential_ttr_p50_s": float(np.percentile(ttr_seq, 50)),
                         "sequential_ttr_p99_s": float(np.percentile(ttr_seq, 99)),
                         "served_makespan_s": t_srv, "sequential_makespan_s": free_at,
                         "peak_active": st["peak_active"],
                         "what": "Poisson arrivals, sizes log-uniform 64^2..200^3 (2-D pack or 3-D GRF), angle "
                                 "from seed 11, steps 50-1000 (1/20 of the workload's), MRT FP32; sequential = "
                                 "the same requests queued one at a time on the plain engine (measured solve "
                                 "times, simulated queue)"}
    return out


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


def reduce_ranks(dist, ms: float, n: int, device: str):
    """Whole-job timing over the replicas: the slowest rank's time and the
    sites of all ranks (identity without a process group)."""
    if dist is None:
        return ms, n
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    nt = torch.tensor([float(n)], dtype=torch.float64, device=device)
    dist.all_reduce(nt)
    return float(t.item()), int(nt.item())


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
    tuned = None
    if args.brick != "auto":
        p.brick = _capi.BRICK[args.brick]
    elif not args.no_autotune:
        # the layout autotuner on this lattice (outside the timed region); the
        # engine below (brick "auto") takes its choice
        from felbm_gpu_b200.engine import autotune
        tuned = autotune(p, solid, steps=30, device=lrank)
    eng = MultiPhaseGPU(p, solid, device=lrank)
    n = eng.n
    brick, graph_steps = eng.layout()
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
    ms, n_total = reduce_ranks(dist, ms, n, "cuda")
    value = n_total * args.steps / (ms / 1e3) / 1e6
    # per-kernel device times (plain launches, CUDA events on the engine stream)
    kms = eng.time_kernels(max(10, min(args.steps, 50))) / max(10, min(args.steps, 50))
    peak, peak_kind = measured_peak()
    t_p4 = kms[4] / 1e3
    achieved = B_P4[args.storage] * n / t_p4 / 1e9
    tr = profiled_traffic(args.storage, args.size, brick)
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
        # statistics of every step come back device->host through the
        # asynchronous form, flow_stats_launch / _collect: step t's are
        # collected once step t+1 is queued, so the device does not idle
        # while the host reads them), and the final state comes back
        # (fe_download_state). Host wall clock around all of it.
        ke = args.steps
        # the caller's host buffers for the result, as a driver holds them
        hd = np.empty_like(h0)
        gd = np.empty_like(g0)
        hd.fill(0.0)
        gd.fill(0.0)
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        eng.upload_state(h0, g0)
        eng.record_target_mass()
        for t in range(ke):
            eng.set_forcing_factor(1.0)
            eng.step(1)
            eng.apply_mass_correction(want_drift=False)
            if t:
                eng.flow_stats_collect()  # step t-1's, read while step t runs
            eng.flow_stats_launch()
        eng.flow_stats_collect()
        eng.download_state(hd, gd)
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
                       "fe_apply_mass_correction, fe_flow_stats_launch, and step t-1's "
                       "fe_flow_stats_collect) + fe_download_state, host wall clock"}
    production = None
    if not args.no_tracers:
        # the production loop: 12,000 GPU tracers (diffusivity ladder
        # 1e-5..1e-1, uniform in the fluid) advanced after every step, flow
        # statistics every 100 steps; device synchronised around the loop
        from felbm_gpu_b200.tracers import Tracers, seed
        pos, _ = seed(solid, 12000, rng_seed=17)
        tr = Tracers(eng, pos, np.logspace(-5, -1, 12000), rng_seed=3)
        for _ in range(3):
            eng.run(1)
            tr.step()
        kp = max(100, (args.steps // 100) * 100)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for s in range(1, kp + 1):
            eng.run(1)
            tr.step()
            if s % 100 == 0:
                eng.flow_stats()
        tr.download()
        torch.cuda.synchronize()
        dtp = time.perf_counter() - t0
        tr.free()
        production = {"workload": "the benched lattice + 12,000 tracers (Dm ladder 1e-5..1e-1), flow statistics "
                                  "every 100 steps; driver loop fe_run(1) + fe_tracers_step per step",
                      "steps": kp, "mlups": n * kp / dtp / 1e6, "ms_per_step": dtp * 1e3 / kp,
                      "tracer_ms_per_step": dtp * 1e3 / kp - ms / args.steps}
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_sample_mlups(args.storage)
    serving = None
    if ws == 1 and not args.no_serve:
        eng.free()
        serving = serve_legs(args)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": args.storage, "data": "synthetic",
                "config": {"workload": f"{args.size}^3 GRF porous (corr 6, porosity 0.37, largest cluster), "
                                       f"periodic, body force 1e-6, fused MRT, theta 45, correct_op_mass, "
                                       f"slab IC, {args.storage} populations",
                           "sites": int(n), "porosity": por, "parallelism": f"replicas x{ws}",
                           "l2": "inputs larger than L2 (state > 1 GB), no flush",
                           "layout": {"brick": brick, "graph_steps": graph_steps,
                                      "autotune": tuned["candidates"] if tuned else None}},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
                "clocks": clk.summary(), "production": production, "serving": serving}
        print(json.dumps(line), flush=True)
    eng.free()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
