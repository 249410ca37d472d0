"""Benchmark: HMC link-updates/s on one B200 (or N independent replicas).

Workload (default ``su3_32``): SU(3) Wilson action, DIM=4, lattice 32^4
(1,048,576 sites, 4,194,304 links), BETA=6.0, DT=0.02, LEVEL=6, 50 leapfrog
steps per trajectory, Haar-random hot start, seeded synthetic data.

A bench "step" is one whole HMC trajectory on the device: momentum refresh,
FP64 H_old, 50 fused kick+drift link updates, closing half kick, FP64 H_new,
Metropolis and the accept/reject copy, replayed as one CUDA graph.
``value`` = link updates per second over the timed trajectories
(links x MD steps x trajectories / device time), aggregated over all ranks.
The headline path is FP32-mixed (FP32 links, reunitarised, FP64 dH); the
plain FP64 path is timed on the same workload and reported beside it.

``e2e`` measures the same metric through the public C ABI with host buffers:
every step uploads the configuration from pinned host memory
(askja_set_links, U-conf layout FP64) and reads the trajectory result back.

``--impl reference`` times the reference's own CPU code (sun.cpp's
updateUandcopyDown + updateE, compiled from the reference sources against the
project's GSL shim into oracle/_ref) on the host cores, one MD step of the
same lattice per bench step; without that build it falls back to the
project's C restatement (oracle/askja_oracle.c).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    # name: nc, dims, beta, dt, level, md steps per trajectory
    "su3_32": dict(nc=3, dims=[32, 32, 32, 32], beta=6.0, dt=0.02, level=6, nsteps=50),
    "su8_10": dict(nc=8, dims=[10, 10, 10, 10], beta=20.0, dt=0.01, level=8, nsteps=100, ensemble=60),
    "su3_8": dict(nc=3, dims=[8, 8, 8, 8], beta=5.70, dt=0.02, level=8, nsteps=50),
    # large NC: every complex product of the FP32 path on the tensor cores (split TF32 x 3);
    # the CPU sample runs the same colour number on a smaller lattice (per-link rates)
    "su32_8": dict(nc=32, dims=[8, 8, 8, 8], beta=2048.0, dt=0.005, level=8, nsteps=20, tensor=True,
                   cpu_dims=[2, 2, 2, 2], ensemble=20),
    "su64_4x16": dict(nc=64, dims=[4, 16, 16], beta=8192.0, dt=0.005, level=8, nsteps=20, tensor=True,
                      cpu_dims=[2, 2, 4], ensemble=20),
    # NC = 16: the tensor cores on the padded M = 64 shape against the row kernels (the autotuner picks)
    "su16_6": dict(nc=16, dims=[6, 6, 6, 6], beta=512.0, dt=0.005, level=8, nsteps=20, tensor=True,
                   cpu_dims=[2, 2, 2, 2], ensemble=20),
}

BATCH_CONFIGS = ("batch64", "batch_su3_32")


def metric_for(config: str) -> str:
    """The metric string of a workload, identical in both arms (ours and
    --impl reference) so that their values can be divided."""
    if config == "batch_su3_32":
        return "link-updates/s (1 B200): HMC, 4 chains SU(3) DIM=4 32x32x32x32, 50 MD steps/trajectory"
    if config == "batch64":
        return "link-updates/s (1 B200): HMC, 64 uneven chains NC 2-8, DIM 2-4, 20 MD steps/trajectory"
    cfg = CONFIGS[config]
    return (f"link-updates/s (1 B200): HMC, SU({cfg['nc']}) DIM={len(cfg['dims'])} "
            f"{'x'.join(map(str, cfg['dims']))}, {cfg['nsteps']} MD steps/trajectory")


PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
FALLBACK_BF16_TFLOPS = 1590.0


def peaks():
    try:
        with open(PEAKS_PATH) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def tf32_peak():
    """Dense TF32 tensor peak: half the measured dense BF16 GEMM rate (the
    tensor cores run TF32 at half the BF16 rate)."""
    try:
        with open(PEAKS_PATH) as f:
            return 0.5 * float(json.load(f)["bf16_tflops"]), "measured bf16 / 2"
    except Exception:
        return 0.5 * FALLBACK_BF16_TFLOPS, "fallback bf16 / 2"


def fp32_peak(device):
    """Measured FP32 FFMA peak of the device, TFLOP/s (askja_peak_flops of the
    bench-only helper library askja_b200/libaskja_peak.so)."""
    import ctypes

    lib = ctypes.CDLL(os.path.join(ROOT, "askja_b200", "libaskja_peak.so"))
    lib.askja_peak_flops.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    g = ctypes.c_double()
    rc = lib.askja_peak_flops(int(device), 0, 5, ctypes.byref(g))
    return g.value / 1e3 if rc == 0 else float("nan")


def link_update_bytes(nc, residual):
    """Compulsory HBM bytes of one fused kick+drift link update in FP32 (neighbour
    links counted as cache hits): read and write the link and its momentum.
    FP32-only storage: 4 x NC^2 complex floats.  Residual-plane mode: the link
    as NC^2 (float2 + bfloat16 pair) = 12 NC^2 bytes, the momentum as NC^2 - 1
    FP32 coordinates plus their bfloat16 residuals in ceil((NC^2 - 1) / 2)
    words; SU(3): 2 x (108 + 48) = 312 bytes."""
    if not residual:
        return 4 * nc * nc * 8
    ncoef = nc * nc - 1
    return 2 * (12 * nc * nc + 4 * ncoef + 4 * ((ncoef + 1) // 2))


def tensor_products_per_link(dim, level, reunit=True):
    """Complex NC x NC products of one fused kick+drift link update on the
    tensor path: 4(D-1) staple products, U S, LEVEL-1 Horner products, E U
    and two Newton-Schulz products."""
    order = level if 0 <= level <= 8 else 8
    return 4 * (dim - 1) + 1 + max(order - 1, 0) + 1 + (2 if reunit else 0)


def tensor_flops_per_link(nc, dim, level, reunit=True):
    """Real MMA flops of one link update on the tensor path: every complex
    product is 2 parts x 3 split pairs of an M=2NC, N=NC, K=NC real MMA."""
    return tensor_products_per_link(dim, level, reunit) * 6 * 2 * (2 * nc) * nc * nc


class Clocks:
    """nvidia-smi sampling during the timed region (every 200 ms)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        if self.path and os.path.exists(self.path):
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _all_reduce(x: float, op: str) -> float:
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(x: float, world: int) -> float:
    """The slowest rank's time: the job is as fast as its slowest replica."""
    return x if world == 1 else _all_reduce(x, "max")


def sum_over_ranks(x: float, world: int) -> float:
    return x if world == 1 else _all_reduce(x, "sum")


def aggregate_rate(units_per_rank: float, world: int, seconds_max: float) -> float:
    """Whole-job throughput: every rank processes `units_per_rank`, the job
    takes the max over ranks of the device time."""
    return units_per_rank * world / seconds_max


def event_timer(stream_ptr: int, device: int):
    import torch
    s = torch.cuda.ExternalStream(stream_ptr, device=device)
    return s, torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def time_trajectories(e, stream_ptr, device, nsteps, steps, warmup, world, clocks=None):
    """W untimed trajectories, then K timed ones (graph replays) bracketed by
    barrier + synchronize; CUDA events on the engine's stream."""
    import torch
    e.run_trajectories(warmup, nsteps, use_graph=True, want_log=False)
    s, t0, t1 = event_timer(stream_ptr, device)
    barrier(world)
    torch.cuda.synchronize()
    e.sync()
    ctx = clocks if clocks is not None else _Null()
    with ctx:
        t0.record(s)
        last, log = e.run_trajectories(steps, nsteps, use_graph=True, want_log=True)
        t1.record(s)
        t1.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    ms = t0.elapsed_time(t1)
    return ms, last, log


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def time_fused_kernel(e, stream_ptr, device, nlaunch, dt):
    """Average duration of one fused kick+drift launch: the slope between
    askja_leapfrog runs of nlaunch and 2 nlaunch fused launches, so that the
    closing kick and the layout conversions around the loop (site-pair
    mapping) cancel."""
    import torch
    s, t0, t1 = event_timer(stream_ptr, device)
    t2 = torch.cuda.Event(enable_timing=True)
    e.leapfrog(2, dt)
    e.sync()
    t0.record(s)
    e.leapfrog(nlaunch, dt)
    t1.record(s)
    e.leapfrog(2 * nlaunch, dt)
    t2.record(s)
    t2.synchronize()
    return (t1.elapsed_time(t2) - t0.elapsed_time(t1)) / nlaunch


def thermalised_links(cfg, ntraj, seed, dev):
    """Haar hot start, then `ntraj` untimed FP32-mixed trajectories (CUDA graph);
    returns the links in U-conf layout (FP64)."""
    import askja_b200 as ab
    with ab.Engine(cfg["nc"], cfg["dims"], beta=cfg["beta"], dt=cfg["dt"], level=cfg["level"], precision="fp32",
                   device=dev, seed=seed + 3) as e:
        e.hot_start(seed + 1)
        if ntraj:
            e.run_trajectories(ntraj, cfg["nsteps"], use_graph=True, want_log=False)
        return e.get_links()


def run_ours(args):
    import torch

    import askja_b200 as ab

    world, rank, local = dist_setup(args.gpus)
    cfg = CONFIGS[args.config]
    nc, dims, nsteps = cfg["nc"], cfg["dims"], cfg["nsteps"]
    vol = int(np.prod(dims))
    links = vol * len(dims)
    dev = local
    torch.cuda.set_device(dev)
    seed = 20240601 + 7919 * rank
    res = {}
    # untimed: Haar hot start, then FP32-mixed trajectories until the chain has left the
    # hot-start transient, so that both timed legs start from the same equilibrated links
    u0 = thermalised_links(cfg, args.therm, seed, dev)
    for prec in ("fp32", "fp64"):
        with ab.Engine(nc, dims, beta=cfg["beta"], dt=cfg["dt"], level=cfg["level"], precision=prec, device=dev,
                       seed=seed) as e:
            e.set_links(u0)
            e.initializeE(seed, 0)
            # untimed: picks the kernel mapping for this (NC, DIM, precision); --no-tune keeps the
            # default mapping (under a profiler the candidates' timings are not representative)
            tuning = {"path": None, "groups": 0, "occupancy": 0, "best_us": None} if args.no_tune \
                else ab.autotune(e, reps=3)
            K = args.steps if prec == "fp32" else max(3, args.steps // 2)
            clocks = Clocks(dev) if prec == "fp32" else None
            ms, last, log = time_trajectories(e, e.stream_ptr, dev, nsteps, K, args.warmup, world, clocks)
            ms_max = max_over_ranks(ms, world)
            lu = aggregate_rate(links * nsteps * K, world, ms_max / 1e3)
            r = dict(ms=ms_max, K=K, lu=lu, acc=last["n_acc"] / max(1, last["n_tot"]),
                     dh_mean=float(np.mean(log[:, 2])), dh_abs=float(np.mean(np.abs(log[:, 2]))),
                     tuning={k: tuning[k] for k in ("path", "groups", "occupancy", "best_us")})
            if clocks is not None:
                r["clocks"] = clocks.summary()
                # dominant kernel: fused kick+drift, timed alone
                r["kernel_ms"] = time_fused_kernel(e, e.stream_ptr, dev, 20, cfg["dt"])
                # e2e through the C ABI with host buffers
                r.update(run_e2e(e, nsteps, max(6, K), world))
                t, s_ = e.PlaqExp()
                r["plaq"] = 1.0 - (t + s_) / (vol * 6)
            res[prec] = r
    if rank != 0:
        return None
    f32, f64 = res["fp32"], res["fp64"]
    hbm, peak_kind = peaks()
    residual = nc <= 4 and not cfg.get("tensor")  # the residual-plane FP32 mode
    # algorithmic bytes of a link update: read U, read P, write P, write U as full
    # NC x NC FP32 complex matrices, neighbour links as cache hits (4 NC^2 x 8 B);
    # the residual planes' own layout moves link_update_bytes (312 B for SU(3))
    alg_per_lu = 4 * nc * nc * 8
    bytes_per_lu = link_update_bytes(nc, residual)
    achieved = alg_per_lu * links / (f32["kernel_ms"] / 1e3) / 1e9
    traffic = measured_traffic(args.config)
    if cfg.get("tensor") and (f32["tuning"]["path"] == 2 or (f32["tuning"]["path"] is None and nc >= 32)):
        fpl = tensor_flops_per_link(nc, len(dims), cfg["level"])
        sec = f32["kernel_ms"] / 1e3
        pk, src = tf32_peak()
        tflops = fpl * links / sec / 1e12
        roofline = {"bound": "tensor", "kernel": f"tensor-core link update (tc::k_link<{nc},1> + per-link copy of U)",
                    "achieved": tflops, "peak": pk, "unit": "TFLOP/s", "frac": tflops / pk, "peak_source": src,
                    "traffic": None, "flops_per_launch": fpl * links, "avg_launch_ms": f32["kernel_ms"],
                    "complex_tflops": 8 * nc ** 3 * tensor_products_per_link(len(dims), cfg["level"]) * links
                    / sec / 1e12}
    elif f32["tuning"]["path"] == 1 or (f32["tuning"]["path"] is None and nc > 4):
        # row-per-thread kernels (NC >= 5): bound by the FP32 FMA pipe; flops per link =
        # 8 NC^3 x (4(D-1) + 1 force products + LEVEL Horner products), against the FFMA peak
        # measured on this device now
        order = cfg["level"] if 0 <= cfg["level"] <= 8 else 8
        fpl = 8 * nc ** 3 * (4 * (len(dims) - 1) + 1 + order)
        pk = fp32_peak(dev)
        tflops = fpl * links / (f32["kernel_ms"] / 1e3) / 1e12
        roofline = {"bound": "fp32", "kernel": f"fused kick+drift (rows::k_force<{nc},float,1>)",
                    "achieved": tflops, "peak": pk, "unit": "TFLOP/s", "frac": tflops / pk,
                    "peak_source": "measured FFMA on this device (askja_peak_flops)", "traffic": None,
                    "flops_per_launch": fpl * links, "avg_launch_ms": f32["kernel_ms"],
                    "hbm_achieved_gbs": achieved}
    else:
        paired = f32["tuning"]["path"] == 3
        kname = ("pair::k_force_pair (site pairs, packed FP32x2)" if paired else
                 f"split::k_force<{nc},1> (FP32 + bfloat16 residual planes)" if residual else
                 f"small::k_force<{nc},float,1>")
        # the FP32 floor beside the HBM one: complex products per link = 4(D-1) + 1 force
        # products + X^2 and (E - 1) U of the Cayley-Hamilton exponential (N <= 3; LEVEL
        # Horner products otherwise), 8 NC^3 flops each, against the FFMA peak measured now
        order = cfg["level"] if 0 <= cfg["level"] <= 8 else 8
        fpl = 8 * nc ** 3 * (4 * (len(dims) - 1) + 1 + (2 if nc <= 3 else order))
        pk32 = fp32_peak(dev)
        tf32 = fpl * links / (f32["kernel_ms"] / 1e3) / 1e12
        roofline = {"bound": "hbm", "kernel": f"fused kick+drift ({kname})",
                    "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                    "peak_source": peak_kind, "traffic": None if paired else traffic,
                    "bytes_per_launch": alg_per_lu * links, "avg_launch_ms": f32["kernel_ms"],
                    "storage_bytes_per_launch": bytes_per_lu * links,
                    "storage_achieved": bytes_per_lu * links / (f32["kernel_ms"] / 1e3) / 1e9,
                    "storage_note": "compulsory bytes of the stored layout (FP32 links and momentum "
                                    "coordinates with bfloat16 residual planes): the traffic to compare "
                                    "`traffic` with",
                    "fp32": {"flops_per_launch": fpl * links, "achieved": tf32, "peak": pk32, "unit": "TFLOP/s",
                             "frac": tf32 / pk32,
                             "peak_source": "measured FFMA on this device (askja_peak_flops)",
                             "note": "matrix-product flops this kernel performs (Cayley-Hamilton scalars, "
                                     "projection, reunitarisation not counted)",
                             # the reference algorithm's count, 8 N^3 (4D + L - 2): L Horner products + E U
                             "reference_algorithm_flops_per_launch": 8 * nc ** 3 * (4 * len(dims) + order - 2) * links,
                             "frac_reference_algorithm": 8 * nc ** 3 * (4 * len(dims) + order - 2) * links
                             / (f32["kernel_ms"] / 1e3) / 1e12 / pk32}}
    field_mb = links * nc * nc * 8 / 1e6
    line = {
        "metric": metric_for(args.config),
        "value": f32["lu"],
        "unit": "link-updates/s",
        "n_gpus": world,
        "steps": f32["K"],
        "warmup": args.warmup,
        "ms_per_step": f32["ms"] / f32["K"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp32 (links, complex) / fp64 (dH, Metropolis)",
        "data": f"synthetic: seeded Haar hot start, {args.therm} untimed FP32 thermalisation trajectories, "
                "Philox momenta",
        "config": {"workload": f"{args.config}: SU({nc}) DIM={len(dims)} {'x'.join(map(str, dims))}, "
                               f"BETA={cfg['beta']}, DT={cfg['dt']}, LEVEL={cfg['level']}, "
                               f"{nsteps} MD steps/trajectory, 1 step = 1 trajectory",
                   "thermalisation_trajectories": args.therm,
                   "links": links, "md_steps_per_traj": nsteps, "parallelism": f"replicas x{world}",
                   "l2": f"links {field_mb:.0f} MB FP32 / {2 * field_mb:.0f} MB FP64 per field; "
                         f"{'inputs larger than L2' if 2 * field_mb > 126 else 'fields partly L2-resident'}"},
        "trajectories_per_s": world * f32["K"] / (f32["ms"] / 1e3),
        "fp64": {"value": f64["lu"], "ms_per_step": f64["ms"] / f64["K"], "steps": f64["K"],
                 "acceptance": f64["acc"], "mean_abs_dH": f64["dh_abs"]},
        "mixed_over_fp64": f32["lu"] / f64["lu"],
        "tuning": {"fp32": f32["tuning"], "fp64": f64["tuning"]},
        "acceptance": f32["acc"],
        "mean_abs_dH": f32["dh_abs"],
        "plaquette": f32["plaq"],
        "e2e": {"value": f32["e2e_lu"], "unit": "link-updates/s", "h2d_bytes_per_step": f32["h2d"],
                "d2h_bytes_per_step": f32["d2h"], "steps": f32["e2e_K"],
                "api": "askja_set_links_async (FP64 U-conf from pinned host memory) + askja_trajectory_async "
                       "(outcome to pinned host memory) per trajectory; uploads overlap the previous trajectory"},
        "roofline": roofline,
        "gpu_launches": f32["K"] * (nsteps + 15) + f64["K"] * (nsteps + 15),
        "clocks": f32["clocks"],
    }
    if args.config == "su3_32" and not args.no_batch:
        # the batched path: FP32-mixed chains batched in one engine vs each chain alone in FP64
        b = run_batch(argparse.Namespace(config="batch_su3_32", steps=max(3, args.steps // 2), warmup=args.warmup,
                                         therm=args.batch_therm))
        line["batched"] = {k: b[k] for k in ("metric", "value", "unit", "steps", "ms_per_step", "alone_fp64",
                                             "alone_fp32", "batched_over_alone_fp64", "batched_over_alone_fp32",
                                             "acceptance_mean", "acceptance_min", "clocks")}
        line["batched"]["workload"] = b["config"]["workload"]
    if not args.no_precision:
        line["precision"] = precision_report(cfg, dev)
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(cfg, args.cpu_md_steps)
    return line


def precision_report(cfg, dev):
    """FP32-mixed vs FP64 on identical (U, P) after a short FP32 thermalisation
    from the hot start: force error, per-trajectory |dH32 - dH64|,
    reversibility and unitarity (askja_b200.precision)."""
    from askja_b200 import precision
    nc, dims = cfg["nc"], cfg["dims"]
    therm = 200
    u0 = precision.thermalise(nc, dims, cfg["beta"], cfg["dt"], cfg["level"], cfg["nsteps"], therm, 4242, dev)
    r = precision.compare(nc, dims, cfg["beta"], cfg["dt"], cfg["level"], cfg["nsteps"], u0, ntraj_dh=3,
                          device=dev)
    r["thermalisation_trajectories"] = therm
    if cfg.get("ensemble"):
        # observables of independent FP32 and FP64 chains from the same start
        r["ensemble"] = precision.ensemble(nc, dims, cfg["beta"], cfg["dt"], cfg["level"], cfg["nsteps"], u0,
                                           ntraj=cfg["ensemble"], device=dev)
    return r


def measured_traffic(config: str):
    """DRAM bytes (read + write) per launch of the fused kernel (residual-plane
    mode) from the committed ncu summary of the same workload, or None."""
    import re
    path = os.path.join(ROOT, "profiles", "fused_kick_drift_su3_32x4.md")
    if config != "su3_32" or not os.path.exists(path):
        return None
    m = re.search(r"traffic_bytes_per_launch_residual_su3_32:\s*(\d+)", open(path).read())
    return int(m.group(1)) if m else None


def run_e2e(e, nsteps, K, world):
    """Same metric through the C ABI with host buffers.  Every trajectory's
    starting configuration (FP64 U-conf layout, the reference's interchange
    format) is uploaded from pinned host memory with askja_set_links_async
    (two host buffers used in turn) and its outcome (askja_traj_result) read
    back to pinned host memory with askja_trajectory_async, so the upload for
    trajectory k+1 runs on the copy engine while trajectory k computes.  Timed
    on the host from the first upload to the synchronisation after the last
    read-back."""
    import ctypes

    import askja_b200 as ab
    nbytes = int(np.prod(e.shape)) * 16
    rsz = ctypes.sizeof(ab.TrajResult)
    bufs = [ab.PinnedBuffer.alloc(nbytes) for _ in range(2)]
    res = ab.PinnedBuffer.alloc(rsz * (K + 1))
    try:
        u = e.get_links()
        for b in bufs:
            b.array(np.complex128, e.shape)[...] = u
        # untimed: staging buffers, graph capture
        e.set_links_async(bufs[0].ptr)
        e.trajectory_async(nsteps, res.ptr + K * rsz)
        e.sync()
        barrier(world)
        t0 = time.perf_counter()
        for k in range(K):
            e.set_links_async(bufs[k % 2].ptr)
            e.trajectory_async(nsteps, res.ptr + k * rsz)
        e.sync()
        dt = time.perf_counter() - t0
        outs = [ab.TrajResult.from_address(res.ptr + k * rsz).as_dict() for k in range(K)]
        assert all(np.isfinite(o["dh"]) for o in outs)
        assert [o["n_tot"] for o in outs] == sorted(o["n_tot"] for o in outs)
    finally:
        for b in bufs:
            b.free()
        res.free()
    dt = max_over_ranks(dt, world)
    links = e.vol * e.dim
    return {"e2e_lu": aggregate_rate(links * nsteps * K, world, dt), "h2d": nbytes, "d2h": rsz, "e2e_K": K}


def cpu_baseline(cfg, md_steps):
    """The reference's own CPU code on this host, one bounded sample."""
    line = run_reference_sample(cfg, md_steps, warmup=0)
    return line


def run_reference_sample(cfg, steps, warmup):
    from oracle import Reference, Oracle, fields
    nc, dims = cfg["nc"], cfg.get("cpu_dims", cfg["dims"])
    cores = os.cpu_count() or 1
    rng = np.random.default_rng(1)
    vol = int(np.prod(dims))
    links = vol * len(dims)
    u = fields.haar(nc, links, rng).reshape(vol, len(dims), nc, nc)
    O = Oracle(nc, dims)
    p = fields.momenta(nc, links, cfg["beta"], rng, O)
    if Reference.available():
        R = Reference(nc, dims, beta=cfg["beta"], level=cfg["level"])
        R.threads(cores)
        R.set("u", u)
        R.set("U", u)
        R.set("pi", p)
        R.set("Pi", p)
        kind = "reference"

        def step():
            R.updateUandcopyDown(cfg["dt"])
            R.updateE(cfg["dt"])
    else:
        kind = "port"
        state = {"u": u, "p": p}

        def step():
            state["u"] = O.updateU(state["u"], state["p"], cfg["dt"], cfg["level"])
            state["p"] = O.updateE(state["u"], state["p"], cfg["dt"])
    for _ in range(warmup):
        step()
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    per = float(np.mean(times))
    return {"value": links / per, "unit": "link-updates/s", "cores": cores, "kind": kind,
            "sample": f"{steps} MD step(s) (updateUandcopyDown + updateE) of SU({nc}) "
                      f"{'x'.join(map(str, dims))}, OMP threads={cores}",
            "seconds_per_md_step": per, "times": times}


def run_reference_chains(chains, steps, warmup):
    """The reference CPU code over every chain of a batch in turn (one MD step
    of each per bench step): aggregate link-updates/s."""
    tot_links, tot_s, parts = 0, 0.0, []
    for c in chains:
        cfg = dict(nc=c["nc"], dims=c["dims"], beta=c["beta"], dt=c["dt"], level=c["level"])
        r = run_reference_sample(cfg, steps, warmup)
        links = int(np.prod(c["dims"])) * len(c["dims"])
        tot_links += links
        tot_s += r["seconds_per_md_step"]
        parts.append(r)
    return {"value": tot_links / tot_s, "unit": "link-updates/s", "cores": parts[0]["cores"], "kind": parts[0]["kind"],
            "sample": f"{steps} MD step(s) of each of the {len(chains)} chains in turn, OMP threads={parts[0]['cores']}",
            "seconds_per_md_step": tot_s}


def batch_chains(n=64, seed=7):
    """64 uneven chains: NC cycling over {2,3,4,8}, DIM over {2,3,4}, extents
    16^2 .. 16^4 (incl. 4x16^3), BETA uniform over [2,4] * NC^2/3."""
    rng = np.random.default_rng(seed)
    shapes = {2: [[16, 16], [8, 16], [16, 8]], 3: [[16, 16, 16], [4, 16, 16], [8, 8, 8]],
              4: [[16, 16, 16, 16], [4, 16, 16, 16], [8, 8, 8, 8], [4, 8, 8, 8]]}
    chains = []
    for i in range(n):
        nc = (2, 3, 4, 8)[i % 4]
        dim = (2, 3, 4)[(i // 4) % 3]
        dims = shapes[dim][(i // 12) % len(shapes[dim])]
        beta = float(rng.uniform(2.0, 4.0) * nc * nc / 3.0)
        chains.append(dict(nc=nc, dims=list(dims), beta=beta, dt=0.1 / np.sqrt(beta), level=8, seed=1000 + i))
    return chains


def batch_su3_32_chains():
    """Four SU(3) 32^4 chains, a beta scan (5.85 .. 6.15) at the headline
    volume: DT 0.02, LEVEL 6 as the single-chain workload."""
    return [dict(nc=3, dims=[32] * 4, beta=b, dt=0.02, level=6, seed=2000 + i)
            for i, b in enumerate((5.85, 5.95, 6.05, 6.15))]


def tune_dt(chains, nsteps, rounds=3, ntraj=6, dev=0):
    """Adjust each chain's DT towards ~80 % acceptance (FP32 batch, untimed)."""
    import askja_b200 as ab
    for _ in range(rounds):
        with ab.Batch(chains, precision="fp32", device=dev) as b:
            b.hot_start(3)
            b.run(4, nsteps)  # leave the hot-start transient
            before = b.run(0, nsteps)
            res = b.run(ntraj, nsteps)
        for c, r, r0 in zip(chains, res, before):
            acc = (r["n_acc"] - r0["n_acc"]) / max(1, r["n_tot"] - r0["n_tot"])
            if acc < 0.65:
                c["dt"] *= 0.75
            elif acc > 0.92:
                c["dt"] *= 1.25
    return chains


def run_batch(args):
    """Configs 'batch64' and 'batch_su3_32': all chains in one batch
    (FP32-mixed) vs each chain alone in FP64 (and FP32) through the
    single-chain engine."""
    import torch

    import askja_b200 as ab
    dev = 0
    torch.cuda.set_device(dev)
    su3 = args.config == "batch_su3_32"
    nsteps = 50 if su3 else 20
    chains = batch_su3_32_chains() if su3 else tune_dt(batch_chains(), nsteps, dev=dev)
    work = sum(int(np.prod(c["dims"])) * len(c["dims"]) for c in chains) * nsteps
    therm = getattr(args, "therm", 0)
    with ab.Batch(chains, precision="fp32", device=dev) as b:
        b.hot_start(5)
        b.run(therm, nsteps)  # untimed thermalisation
        start = [b.get_links(c) for c in range(len(chains))]
        b.run(args.warmup, nsteps)
        s, t0, t1 = event_timer(b.stream_ptr, dev)
        torch.cuda.synchronize()
        r0 = b.run(0, nsteps)
        with Clocks(dev) as clocks:
            t0.record(s)
            res = b.run(args.steps, nsteps)
            t1.record(s)
            t1.synchronize()
        ms = t0.elapsed_time(t1)
        acc = [(r["n_acc"] - a["n_acc"]) / max(1, r["n_tot"] - a["n_tot"]) for r, a in zip(res, r0)]
    batched = work * args.steps / (ms / 1e3)
    # each chain alone (single-chain engine, CUDA graph), FP64 and FP32
    alone = {}
    for prec in ("fp64", "fp32"):
        tot_ms = 0.0
        for ci, c in enumerate(chains):
            with ab.Engine(c["nc"], c["dims"], beta=c["beta"], dt=c["dt"], level=c["level"], precision=prec,
                           device=dev, seed=c["seed"]) as e:
                e.set_links(start[ci])
                e.run_trajectories(2, nsteps, use_graph=True, want_log=False)
                s, a, z = event_timer(e.stream_ptr, dev)
                e.sync()
                a.record(s)
                e.run_trajectories(args.steps, nsteps, use_graph=True, want_log=False)
                z.record(s)
                z.synchronize()
                tot_ms += a.elapsed_time(z)
        alone[prec] = work * args.steps / (tot_ms / 1e3)
    metric = metric_for(args.config)
    if su3:
        workload = (f"batch_su3_32: 4 chains SU(3) DIM=4 32^4, BETA 5.85/5.95/6.05/6.15, DT=0.02, LEVEL=6, "
                    f"{nsteps} MD steps/trajectory, {therm} untimed thermalisation trajectories, "
                    "1 step = 1 trajectory of every chain, FP32-mixed batched vs each chain alone in FP64")
    else:
        workload = ("batch64: NC in {2,3,4,8}, DIM in {2,3,4}, 16^2..16^4 incl. 4x16^3, "
                    f"BETA in [2,4]*NC^2/3, {nsteps} MD steps/trajectory, DT tuned per chain, "
                    f"{therm} untimed thermalisation trajectories, "
                    "1 step = 1 trajectory of every chain, FP32-mixed batched vs each chain alone in FP64")
    return {
        "metric": metric,
        "value": batched, "unit": "link-updates/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32 (links) / fp64 (dH)", "data": "synthetic: Haar hot start, Philox momenta",
        "config": {"workload": workload, "chains": len(chains), "links_total": work // nsteps},
        "alone_fp64": alone["fp64"], "alone_fp32": alone["fp32"],
        "batched_over_alone_fp64": batched / alone["fp64"],
        "batched_over_alone_fp32": batched / alone["fp32"],
        "acceptance_mean": float(np.mean(acc)), "acceptance_min": float(np.min(acc)),
        "clocks": clocks.summary(),
    }


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    if args.config == "batch64":
        r = run_reference_chains(batch_chains(), args.steps, args.warmup)
        workload = "batch64: each of the 64 chains in turn"
    else:
        cfg = CONFIGS["su3_32" if args.config == "batch_su3_32" else args.config]
        r = run_reference_sample(cfg, args.steps, args.warmup)
        nc, dims = cfg["nc"], cfg.get("cpu_dims", cfg["dims"])
        workload = f"{args.config}: SU({nc}) DIM={len(dims)} {'x'.join(map(str, dims))}"
    line = {
        "impl": "reference",
        "metric": metric_for(args.config),
        "value": r["value"], "unit": "link-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["seconds_per_md_step"] * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp64", "data": "synthetic: seeded Haar links",
        "config": {"workload": f"{workload}; 1 step = 1 MD step of the reference CPU code",
                   "parallelism": "CPU OpenMP"},
        "cpu_baseline": {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": r["value"], "unit": "link-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


def run_kernel_only(args):
    """Kernel microbenchmark (also the command the ncu summaries under
    profiles/ capture): one engine of the config, Haar hot start, Philox
    momenta, `--warmup` single-step leapfrogs, then askja_leapfrog runs of 2,
    `--steps` and 2 `--steps` fused kick+drift launches (each + 1 kick) with
    the default (untuned) kernel mapping or the one `--path` forces.  Prints
    the launch time from the slope between the last two runs."""
    import torch

    import askja_b200 as ab
    cfg = CONFIGS[args.config]
    nc, dims = cfg["nc"], cfg["dims"]
    with ab.Engine(nc, dims, beta=cfg["beta"], dt=cfg["dt"], level=cfg["level"], precision=args.precision,
                   kernel_path=args.path) as e:
        if args.occ or args.groups:
            ab.set_tuning(e, {"path": args.path, "occupancy": args.occ, "groups": args.groups})
        e.hot_start(11)
        e.initializeE(11, 0)
        for _ in range(args.warmup):
            e.leapfrog(1, cfg["dt"])
        e.sync()
        ms = time_fused_kernel(e, e.stream_ptr, 0, args.steps, cfg["dt"])
    return {"kernel_only": args.config, "precision": args.precision, "path": args.path, "occ": args.occ,
            "groups": args.groups,
            "launches": 3 * args.steps + 2, "avg_launch_ms": ms,
            "link_updates_per_s": int(np.prod(dims)) * len(dims) / (ms / 1e3)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="su3_32", choices=sorted(CONFIGS) + list(BATCH_CONFIGS))
    ap.add_argument("--cpu-md-steps", type=int, default=2)
    ap.add_argument("--therm", type=int, default=100, help="untimed FP32 thermalisation trajectories before timing")
    ap.add_argument("--batch-therm", type=int, default=50, help="untimed thermalisation of the batched sub-run")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched sub-run of the default line")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-precision", action="store_true")
    ap.add_argument("--kernel-only", action="store_true", help="fused-kernel microbenchmark (profiling)")
    ap.add_argument("--no-tune", action="store_true", help="default kernel mapping, no autotuning")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp32-lean", "fp64"], help="with --kernel-only")
    ap.add_argument("--path", type=int, default=0, help="with --kernel-only: askja kernel_path")
    ap.add_argument("--occ", type=int, default=0, help="with --kernel-only: register budget (askja_tuning.occupancy)")
    ap.add_argument("--groups", type=int, default=0, help="with --kernel-only: askja_tuning.groups")
    args = ap.parse_args()
    if args.kernel_only:
        line = run_kernel_only(args)
    elif args.impl == "reference":
        line = run_reference(args)
    elif args.config in BATCH_CONFIGS:
        args.therm = args.batch_therm
        line = run_batch(args)
    else:
        line = run_ours(args)
    if line is not None:
        print(json.dumps(line), flush=True)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1 and args.impl == "ours":
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
