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
                   tree), on the same 300^3 lattice, same seed and parameters.
                   Its process never loads the engine library: the lattice
                   and the order parameter are built by a child process and
                   handed over as arrays.

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
    ap.add_argument("--pop-layout", default="two_buffers", choices=["two_buffers", "in_place"],
                    help="population layout of the benched engine (in_place: one buffer, AA pattern)")
    ap.add_argument("--sweep-steps", type=int, default=5000, help="steps per solve of the 64-solve sweep")
    ap.add_argument("--stream-seconds", type=float, default=15.0, help="arrival window of the request stream")
    ap.add_argument("--stream-rate", type=float, default=4.0, help="Poisson arrival rate (requests / s)")
    ap.add_argument("--e2e-steps", type=int, default=500,
                    help="steps of the end-to-end job (one state upload and download per job)")
    ap.add_argument("--no-ref-kernels", action="store_true",
                    help="skip timing the reference's own kernels on this GPU")
    ap.add_argument("--precision-study", action="store_true",
                    help="also run every storage type against FP64 on the precision configuration")
    ap.add_argument("--seed", type=int, default=2024, help="seed of the random-field lattice (rank r adds r)")
    ap.add_argument("--emit-workload", default=None, help=argparse.SUPPRESS)
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    lrank = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, lrank


def workload(size: int, seed: int = 2024, **over):
    """The production dispersion configuration: fluid physics of the
    reference's cfg/3d_image/params.cfg (rho0 = rho1 = 1, tau = 0.9, W = 5,
    sigma = 0.0083, mobility_coeff 0.02) with a 45 degree contact angle
    (phi = 6 sigma cos 45) and body force 1e-6 along x, on a random field
    (correlation length 6) at porosity 0.37, largest x-spanning cluster,
    periodic, mass correction, slab start. Keyword overrides go to the
    physics parameters."""
    from felbm_gpu_b200 import default_params, geometry
    shape = (size, size, size)
    solid, por = geometry.grf(shape, 6.0, 0.37, seed, flow_axis=0)
    sigma, W = 0.0083, 5.0
    kw = dict(rho0=1.0, rho1=1.0, tau0=0.9, tau1=0.9, surface_tension=sigma, interface_width=W,
              mobility_coeff=0.02, phi=6 * sigma * np.cos(np.radians(45.0)), gx=1e-6,
              use_mrt=1, use_halfway_bb=1, correct_op_mass=1,
              stream_matrix_free=1, grad_matrix_free=1, fused=1, fuse_collision=1,
              mrt_fast_transform=1, stream_inplace=1)
    kw.update(over)
    p = default_params(**kw)
    c = geometry.order_parameter(solid, "slab", W, origin=(0, 0, 0), axis=0, thickness=size // 2)
    h, g = geometry.equilibrium(c, 1.0, p.rho0, p.rho1)
    return solid, por, p, h, g


def plain_workload(size: int = 200, seed: int = 12345, **over):
    """The plain-method configuration: quasi-2-D size x size x 1, fully
    periodic, random non-overlapping cylinder pack (radii uniform 6-12,
    porosity 0.65), density ratio 1, tau 1 in both phases, W = 4,
    sigma = 1e-3, mobility coefficient 0.02, MRT with s_e = s_eps = 1.19 and
    s_q = 1.2 (nu rates from tau), slab c = 1 for x < size / 2, body force
    1e-6 along x, contact angle 90 degrees (phi = 0), halfway bounce-back."""
    from felbm_gpu_b200 import default_params, geometry
    solid, _ = geometry.cylinders((1, size, size), 6.0, 12.0, 0.65, seed)
    kw = dict(rho0=1.0, rho1=1.0, tau0=1.0, tau1=1.0, surface_tension=1e-3, interface_width=4.0,
              mobility_coeff=0.02, use_mrt=1, use_halfway_bb=1, gx=1e-6, phi=0.0)
    kw.update(over)
    p = default_params(**kw)
    for k, v in ((1, 1.19), (2, 1.19), (3, 1.2)):  # FE_MRT_E, FE_MRT_EPS, FE_MRT_Q fixed
        p.mrt_rate_mode[k] = 2
        p.mrt_rate_value[k] = v
    c = geometry.order_parameter(solid, "slab", 4.0, origin=(0, 0, 0), axis=0, thickness=size // 2)
    h, g = geometry.equilibrium(c, 1.0, p.rho0, p.rho1)
    return solid, p, h, g


def precision_workload(size: int = 150, mrt: bool = True, seed: int = 7, **over):
    """The precision configuration: random-field medium (correlation length
    6, porosity 0.35, largest x-spanning cluster) between open inlet and
    outlet along x (2 empty + 2 buffer layers, copy_to_buffers), pressure
    difference 1e-3 in density units, periodic in y and z, contact angle 60
    degrees, slab start, BGK or MRT. Returns (solid, params, open boundary,
    h, g, porosity)."""
    from felbm_gpu_b200 import OpenBoundary, default_params, geometry
    medium, por = geometry.grf((size, size, size), 6.0, 0.35, seed, flow_axis=0)
    solid = geometry.pad_open(medium, 0, 2, 2)
    inl, outl, bv, br, coord = geometry.open_lists(solid, 0, 2, split_axis=1)
    sigma, W = 1e-3, 4.0
    kw = dict(rho0=1.0, rho1=1.0, tau0=1.0, tau1=1.0, surface_tension=sigma, interface_width=W,
              mobility_coeff=0.02, phi=6 * sigma * np.cos(np.radians(60.0)), use_mrt=int(mrt), use_halfway_bb=1)
    kw.update(over)
    p = default_params(**kw)
    ob = OpenBoundary(inlet=inl, outlet=outl, inlet_coord=coord, buf_verts=bv, buf_refs=br, copy_to_buffers=True,
                      use_in_prs=True, p_in=1.0 + 1e-3 / 3.0, use_out_prs=True, p_out=1.0, use_in_fluid=True,
                      use_out_fluid=True, c_out_fixed=0.0, inlet_c_a=1.0, rho_out_fixed=p.rho1)
    nx = solid.shape[2]
    c = geometry.order_parameter(solid, "slab", W, origin=(0, 0, 0), axis=0, thickness=nx // 2)
    h, g = geometry.equilibrium(c, 1.0, p.rho0, p.rho1)
    return solid, p, ob, h, g, por


def emit_workload(path: str, size: int, seed: int):
    """Child process of the reference arm: the workload's mask, order
    parameter and parameter block into `path` (.npz)."""
    solid, por, p, h, _ = workload(size, seed)
    c = h.reshape(Q, -1).sum(axis=0)  # at rest h_k = w_k c
    np.savez(path, solid=np.packbits(solid.ravel()), shape=np.array(solid.shape), c=c,
             params=np.frombuffer(bytes(p), np.uint8), porosity=np.array(por))


# D3Q19 weights in the velocity order of the C-ABI (rest, 6 axes, 12 edges)
W19 = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)


def workload_without_engine(size: int, seed: int):
    """The workload of workload(size, seed) in a process that must not load
    the engine library: a child process builds it, this one rebuilds the
    rest-state populations h_k = w_k c, g_k = w_k p0 (p0 = 1) in numpy."""
    import tempfile
    from oracle.oracle_py import capi
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "workload.npz")
        subprocess.run([sys.executable, os.path.abspath(__file__), "--emit-workload", path, "--size", str(size),
                        "--seed", str(seed)], check=True)
        z = np.load(path)
        shape = tuple(int(v) for v in z["shape"])
        solid = np.unpackbits(z["solid"], count=int(np.prod(shape))).reshape(shape)
        c = z["c"]
        p = capi.FeParams.from_buffer_copy(z["params"].tobytes())
        por = float(z["porosity"])
    h = (W19[:, None] * c[None, :]).ravel()
    g = np.repeat(W19, c.size)
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


def host_threads() -> int:
    """Host threads this process may run on (the CPU affinity mask, which a
    container's CPU set narrows), the oracle's OpenMP thread count."""
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def oracle_timing(size: int, seed: int, warmup: int, steps: int):
    """The CPU oracle (the reference step restated in C++/OpenMP, FP64) on
    the benched lattice, in this process: `warmup` steps of the reference
    driver loop (forcing factor, step, mass correction), then `steps` timed
    ones, host wall clock, all host threads. This process must not have
    loaded the engine library (the lattice comes from a child process)."""
    from oracle import oracle_py
    from oracle.oracle_py import Oracle
    solid, por, p, h, g = workload_without_engine(size, seed)
    cores = host_threads()
    oracle_py.set_threads(cores)
    o = Oracle(p, solid)
    o.upload_state(h, g)
    del h, g
    o.record_target_mass()
    o.run(warmup, 0)
    t0 = time.perf_counter()
    o.run(steps, warmup)
    dt = time.perf_counter() - t0
    return {"mlups": o.n * steps / dt / 1e6, "seconds": dt, "sites": int(o.n), "cores": oracle_py.threads(),
            "porosity": por, "warmup": warmup, "steps": steps}


def cpu_sample_mlups(size: int, seed: int, warmup: int = 2, steps: int = 8):
    """The reference arm, run as a child process on a bounded sample of the
    same job (a few steps of the same lattice), so that this leg and
    `--impl reference` time the same code in the same kind of process."""
    cmd = [sys.executable, os.path.abspath(__file__), "--impl", "reference", "--size", str(size), "--seed",
           str(seed), "--steps", str(steps), "--warmup", str(warmup)]
    r = subprocess.run(cmd, check=True, capture_output=True, text=True)
    line = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
    cb = dict(line["cpu_baseline"])
    cb["sample"] = (f"the reference arm (--impl reference) as a child process: {steps} timed steps after "
                    f"{warmup} warm-up steps of the benched lattice; " + cb["sample"])
    return cb


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
        srv = Server(storage=storage, chunk_steps=50, latency_first=True)
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
                                 "from seed 11, steps 50-1000 (1/20 of the workload's), MRT FP32; served with "
                                 "latency-first chunks (at most 2 s1 + 131072 sites); sequential = "
                                 "the same requests queued one at a time on the plain engine (measured solve "
                                 "times, simulated queue)"}
    return out


def run_reference_arm(args, ws, rank):
    """The reference's CPU path on this box's host cores, on the benched
    lattice itself (same size, seed, parameters and initial state). Under
    torchrun only rank 0 runs it."""
    if rank != 0:
        return 0
    r = oracle_timing(args.size, args.seed, max(args.warmup, 1), args.steps)
    v = r["mlups"]
    line = {"metric": METRIC, "value": v, "unit": "MLUPS", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["seconds"] * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": f"{args.size}^3 GRF porous (corr 6, porosity 0.37, largest cluster), periodic, "
                                   f"body force 1e-6, fused MRT, theta 45, correct_op_mass, slab IC "
                                   f"(the same lattice, seed and parameters as the engine arm)",
                       "sites": r["sites"], "porosity": r["porosity"], "seed": args.seed},
            "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": r["cores"], "kind": "port",
                             "sample": f"CPU oracle (C++/OpenMP restatement of the reference step, FP64; the "
                                       f"reference's own CPU engine, felbm_local, is not in the reference "
                                       f"snapshot) on the whole {args.size}^3 lattice ({r['sites']} sites): "
                                       f"{r['warmup']} warm-up + {r['steps']} timed steps of the driver loop "
                                       f"(step + mass correction), {r['seconds']:.1f} s, {r['cores']} threads"},
            "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def reference_kernels_leg(solid, p, h0, g0, warmup: int, steps: int, precision: str = "f32"):
    """The reference's own device kernels (include/felbm_gpu/device_engine.cuh,
    compiled unmodified for sm_100a into oracle/_ref/) on this GPU, driven in
    the MultiPhaseGPU::step order on the CPU oracle's neighbour and case
    tables, on the benched lattice: the same-box GPU baseline. Times the
    reference driver loop (step + mass correction, whose host read-back of
    the mass sums blocks every step) and the steps alone, host wall clock
    around queued work with the device synchronised on both sides."""
    from oracle.oracle_py import Oracle
    from oracle.ref_py import RefKernels, available
    if not available(precision):
        return {"unavailable": "oracle/_ref not built (the reference sources were absent at build time)"}
    o = Oracle(p, solid)
    r = RefKernels(p, o, precision=precision)
    n = r.n
    del o
    try:
        r.upload_state(h0, g0)
        r.record_target_mass()
        lib, hd = r.lib, r._h
        for _ in range(warmup):
            lib.ref_step(hd)
            r.apply_mass_correction()
        assert lib.ref_sync() == 0
        t0 = time.perf_counter()
        for _ in range(steps):
            lib.ref_step(hd)
            r.apply_mass_correction()
        assert lib.ref_sync() == 0
        dt_loop = time.perf_counter() - t0
        t0 = time.perf_counter()
        for _ in range(steps):
            lib.ref_step(hd)
        assert lib.ref_sync() == 0
        dt_step = time.perf_counter() - t0
    finally:
        r.close()
    return {"impl": "reference device_engine.cuh kernels, unmodified, sm_100a, all six fast switches on",
            "precision": precision, "sites": int(n), "steps": steps, "warmup": warmup,
            "mlups_step_plus_correction": n * steps / dt_loop / 1e6,
            "ms_per_step_plus_correction": dt_loop * 1e3 / steps,
            "mlups_step": n * steps / dt_step / 1e6, "ms_per_step": dt_step * 1e3 / steps,
            "clock": "host wall clock around queued steps, device synchronised on both sides"}


def interface_area(solid: np.ndarray, c_sites: np.ndarray) -> int:
    """Fluid node pairs along x, y, z (periodic) whose c straddles 1/2."""
    grid = np.full(solid.shape, np.nan)
    grid[solid == 0] = c_sites
    s = grid - 0.5
    n = 0
    for ax in range(3):
        if solid.shape[ax] == 1:
            continue
        t = np.roll(s, -1, axis=ax)
        n += int(np.count_nonzero((s * t) < 0))  # NaN pairs compare False
    return n


def precision_run(solid, p, ob, h, g, storage: str, steps: int, tracers: int = 0, dm: float = 1e-2):
    """One solve in `storage`: fields after `steps`, the mass before and
    after, and (tracers > 0) the longitudinal dispersion coefficient of
    `tracers` tracers of diffusivity dm seeded in the fluid, from the growth
    of the variance of their unwrapped x displacement over the run."""
    import ctypes as C
    from felbm_gpu_b200 import MultiPhaseGPU, _capi
    from felbm_gpu_b200.tracers import Tracers, seed
    q = _capi.FeParams()
    C.pointer(q)[0] = p
    q.storage = _capi.STORAGE[storage]
    e = MultiPhaseGPU(q, solid)
    try:
        if ob is not None:
            e.set_open_bnd(ob)
        e.upload_state(h, g)
        if p.correct_op_mass:
            e.record_target_mass()
        m0 = e.get_target_mass() if p.correct_op_mass else None
        disp = None
        if tracers:
            pos, _ = seed(solid, tracers, rng_seed=5)
            tr = Tracers(e, pos, dm, rng_seed=9)
            nx = solid.shape[2]
            x_prev = tr.download()[0][0].copy()
            dx = np.zeros_like(x_prev)
            done = 0
            while done < steps:
                k = min(10, steps - done)
                for _ in range(k):
                    e.run(1)
                    tr.step()
                done += k
                x = tr.download()[0][0]
                d = x - x_prev
                d -= nx * np.round(d / nx)  # minimal image: a tracer moves < 1 node a step
                dx += d
                x_prev = x.copy()
            disp = float(np.var(dx) / (2.0 * steps))
            tr.free()
        else:
            e.run(steps)
        f = e.download()
        m = e.current_mass() if p.correct_op_mass else None
        return f, m0, m, disp
    finally:
        e.free()


def precision_study(size: int = 150, steps: int = 5000, mass_steps: int = 2000):
    """Every storage type beside FP64 on the precision configuration (open,
    BGK and MRT, `steps`) and on the production configuration at `size`
    (periodic, mass correction, tracers, `mass_steps`): max|dc|, max|du|, the
    relative difference of the interface area, the order-parameter mass
    drift per 1e4 steps and the tracer dispersion coefficient."""
    cases = []
    for mrt in (False, True):
        solid, p, ob, h, g, por = precision_workload(size, mrt)
        cases.append((f"open {size}^3 {'MRT' if mrt else 'BGK'}", solid, p, ob, h, g, por, steps, 0))
    solid, por, p, h, g = workload(size)
    cases.append((f"periodic {size}^3 MRT, mass correction, 4000 tracers", solid, p, None, h, g, por, mass_steps,
                  4000))
    out = []
    for name, solid, p, ob, h, g, por, nsteps, ntr in cases:
        ref, m0, m_ref, d_ref = precision_run(solid, p, ob, h, g, "f64", nsteps, ntr)
        a_ref = interface_area(solid, ref["c"])
        for st in ("f64", "f32", "f16g", "bf16g", "f16s", "bf16s"):
            f, m0s, m, disp = (ref, m0, m_ref, d_ref) if st == "f64" else precision_run(solid, p, ob, h, g, st,
                                                                                         nsteps, ntr)
            du = np.sqrt((f["ux"] - ref["ux"]) ** 2 + (f["uy"] - ref["uy"]) ** 2 + (f["uz"] - ref["uz"]) ** 2)
            area = interface_area(solid, f["c"])
            rec = {"case": name, "storage": st, "steps": nsteps, "sites": int(len(ref["c"])), "porosity": por,
                   "max_abs_dc": float(np.max(np.abs(f["c"] - ref["c"]))), "max_abs_du": float(np.max(du)),
                   "max_abs_u_fp64": float(np.max(np.sqrt(ref["ux"] ** 2 + ref["uy"] ** 2 + ref["uz"] ** 2))),
                   "interface_area": area, "interface_area_rel_diff": (area - a_ref) / a_ref if a_ref else 0.0}
            if m0s is not None:
                rec["mass_drift_rel_per_1e4_steps"] = abs(m - m0s) / abs(m0s) * 1e4 / nsteps
            if disp is not None:
                rec["dispersion_coeff"] = disp
                rec["dispersion_rel_diff"] = (disp - d_ref) / d_ref
            out.append(rec)
    return out


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
    if args.emit_workload:
        emit_workload(args.emit_workload, args.size, args.seed)
        return 0
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
    solid, por, p, h0, g0 = workload(args.size, seed=args.seed + rank)
    p.storage = _capi.STORAGE[args.storage]
    p.pop_layout = 1 if args.pop_layout == "in_place" else 0
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
        # (fe_download_state). Host wall clock around all of it. The job is
        # --e2e-steps long (the production runs are 20,000 steps), at least K.
        ke = max(args.steps, args.e2e_steps)
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
        cpu = cpu_sample_mlups(args.size, args.seed)
    ref_kernels = None
    if rank == 0 and ws == 1 and not args.no_ref_kernels:
        # the reference's kernels need the lattice's FP32 device memory
        # beside ours (about 1.5 KB a site): run them with our engine freed
        eng.free()
        ref_kernels = reference_kernels_leg(solid, p, h0, g0, warmup=max(args.warmup, 3), steps=max(args.steps, 20))
    precision = None
    if rank == 0 and ws == 1 and args.precision_study:
        eng.free()
        precision = precision_study(150)
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
                           "layout": {"brick": brick, "graph_steps": graph_steps, "populations": args.pop_layout,
                                      "autotune": tuned["candidates"] if tuned else None}},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
                "clocks": clk.summary(), "production": production, "serving": serving,
                "reference_kernels": ref_kernels, "precision_study": precision}
        print(json.dumps(line), flush=True)
    eng.free()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
