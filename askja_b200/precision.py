"""Precision of the FP32-mixed engine against the FP64 engine on identical
inputs (same links U and momenta P, both uploaded in FP64 U-conf layout).

Reported quantities:
  force_rel_err     max over links |F32 - F64| / max |F64| for one updateE
  dH                per trajectory: dH of the FP32 path, of the FP64 path and
                    |dH32 - dH64| (both Hamiltonians summed in FP64)
  reversibility     max |U_back - U_0| after nsteps forward, P -> -P,
                    nsteps back (FP32 with reunitarisation, and FP64)
  unitarity         max |U U^dag - 1| of the FP32 links after a trajectory
  ensemble          <plaquette> and <|Polyakov|> over independent FP32 and
                    FP64 Markov chains from the same start, with binned errors

    python -m askja_b200.precision --nc 3 --dims 32 32 32 32 --beta 6.0 --dt 0.02 --level 6 --nsteps 50
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import Engine


def _binned_error(x: np.ndarray, nbins: int = 10) -> float:
    """Standard error of the mean from nbins blocks (absorbs autocorrelation)."""
    x = np.asarray(x, dtype=np.float64)
    n = len(x) // nbins * nbins
    if n < nbins or nbins < 2:
        return float("nan")
    b = x[:n].reshape(nbins, -1).mean(axis=1)
    return float(b.std(ddof=1) / np.sqrt(nbins))


def thermalise(nc, dims, beta, dt, level, nsteps, ntraj, seed, device=0, reunitarise=None, kernel_path=0,
               fp32="fp32"):
    """Hot start, then `ntraj` FP32-mixed trajectories (engine precision `fp32`:
    "fp32" or "fp32-lean"); returns FP64 U-conf links."""
    with Engine(nc, dims, beta=beta, dt=dt, level=level, precision=fp32, device=device, seed=seed,
                reunitarise=reunitarise, kernel_path=kernel_path) as e:
        e.hot_start(seed + 1)
        if ntraj:
            e.run_trajectories(ntraj, nsteps, use_graph=True, want_log=False)
        return e.get_links()


def compare(nc, dims, beta, dt, level, nsteps, u0, ntraj_dh=3, seed=7, device=0, reunitarise=None, kernel_path=0,
            fp32="fp32"):
    out = {}
    kw = dict(beta=beta, dt=dt, level=level, device=device)
    with Engine(nc, dims, precision="fp64", seed=seed, **kw) as e64, \
            Engine(nc, dims, precision=fp32, seed=seed, reunitarise=reunitarise, kernel_path=kernel_path,
                   **kw) as e32:
        # one force evaluation on identical inputs
        e64.set_links(u0)
        e64.initializeE(seed, 12345)
        p0 = e64.get_momenta(0)
        e32.set_links(u0)
        e32.set_momenta(p0, 0)
        e64.updateE(dt)
        e32.updateE(dt)
        f64 = (e64.get_momenta(1) - p0)
        f32 = (e32.get_momenta(1) - p0)
        out["force_rel_err"] = float(np.abs(f32 - f64).max() / np.abs(f64).max())
        # per-trajectory dH on identical (U, P)
        rows = []
        for t in range(ntraj_dh):
            e64.set_links(u0)
            e64.initializeE(seed, 1000 + t)
            p = e64.get_momenta(0)
            e32.set_links(u0)
            e32.set_momenta(p, 0)
            h, ds = [], []
            for e in (e64, e32):
                h0, s0 = e.hamiltonian(0), e.EnergyMag()
                e.leapfrog(nsteps, dt)
                h.append(e.hamiltonian(0) - h0)
                ds.append(beta * (e.EnergyMag() - s0))
            # dS64: the trajectory's change of the action (a relative bias c of
            # the FP32 force shows up as dH32 - dH64 ~ c dS)
            rows.append({"dH64": h[0], "dH32": h[1], "abs_diff": abs(h[1] - h[0]), "dS64": ds[0]})
            if t == 0:
                u32 = e32.get_links().reshape(-1, nc, nc)
                out["unitarity_max"] = float(np.abs(np.einsum("lij,lkj->lik", u32, u32.conj()) - np.eye(nc)).max())
                out["links_max_dev_fp32_vs_fp64"] = float(np.abs(e32.get_links() - e64.get_links()).max())
        out["dH"] = rows
        out["max_abs_dH_diff"] = max(r["abs_diff"] for r in rows)
        out["mean_signed_dH_diff"] = float(np.mean([r["dH32"] - r["dH64"] for r in rows]))
        # reversibility
        rev = {}
        for name, e in (("fp64", e64), ("fp32", e32)):
            e.set_links(u0)
            e.set_momenta(p0, 0)
            e.leapfrog(nsteps, dt)
            e.set_momenta(-e.get_momenta(0), 0)
            e.leapfrog(nsteps, dt)
            rev[name] = float(np.abs(e.get_links() - u0).max())
        out["reversibility"] = rev
    return out


def ensemble(nc, dims, beta, dt, level, nsteps, u0, ntraj, seed=11, device=0, reunitarise=None, kernel_path=0,
             fp32="fp32"):
    res = {}
    vol = int(np.prod(dims))
    D = len(dims)
    nplaq = vol * D * (D - 1) // 2
    nt, ns = vol * (D - 1), vol * (D - 1) * (D - 2) // 2  # temporal (0,k) / spatial (j,k) planes
    obs = ("plaquette", "plaquette_t", "plaquette_s", "polyakov", "wilson")
    for prec in ("fp64", "fp32"):
        extra = dict(reunitarise=reunitarise, kernel_path=kernel_path) if prec == "fp32" else {}
        with Engine(nc, dims, beta=beta, dt=dt, level=level, precision=fp32 if prec == "fp32" else prec,
                    device=device, seed=seed, **extra) as e:
            e.set_links(u0)
            series = {k: [] for k in obs}
            acc = 0
            t0 = time.perf_counter()
            for _ in range(ntraj):
                last, _ = e.run_trajectories(1, nsteps, use_graph=True, want_log=False)
                acc += int(last["accepted"] != 0)
                series["plaquette"].append(1.0 - e.EnergyMag() / nplaq)
                t, s = e.PlaqExp()
                series["plaquette_t"].append(1.0 - t / nt if nt else float("nan"))
                series["plaquette_s"].append(1.0 - s / ns if ns else float("nan"))
                series["polyakov"].append(e.PolyakovLoop())
                series["wilson"].append(e.WilsonLoop())
            r = {"acceptance": acc / max(1, ntraj), "seconds": time.perf_counter() - t0}
            for k in obs:
                r[k] = float(np.mean(series[k]))
                r[k + "_err"] = _binned_error(np.array(series[k]))
            res[prec] = r
    # FP32 minus FP64 for each observable, in units of the combined binned error
    for k in obs:
        d = res["fp32"][k] - res["fp64"][k]
        sig = float(np.hypot(res["fp32"][k + "_err"], res["fp64"][k + "_err"]))
        res[k + "_diff"] = d
        res[k + "_diff_in_sigma"] = float(abs(d) / sig) if sig > 0 else float("inf")
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nc", type=int, default=3)
    ap.add_argument("--dims", type=int, nargs="+", default=[32, 32, 32, 32])
    ap.add_argument("--beta", type=float, default=6.0)
    ap.add_argument("--dt", type=float, default=0.02)
    ap.add_argument("--level", type=int, default=6)
    ap.add_argument("--nsteps", type=int, default=50)
    ap.add_argument("--therm", type=int, default=100)
    ap.add_argument("--dh-traj", type=int, default=5)
    ap.add_argument("--ensemble", type=int, default=0, help="trajectories per precision for <plaq>, <|P|>")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--fp32-reunit", choices=["default", "on", "off"], default="default",
                    help="FP32 engines: per-update reunitarisation (default: on)")
    ap.add_argument("--fp32-path", type=int, default=0, help="FP32 engines: askja kernel_path")
    ap.add_argument("--fp32-storage", choices=["residual", "lean"], default="residual",
                    help="FP32 engines: FP32 + bfloat16 residual planes, or FP32-only storage")
    a = ap.parse_args()
    kw = dict(reunitarise={"default": None, "on": True, "off": False}[a.fp32_reunit], kernel_path=a.fp32_path,
              fp32="fp32" if a.fp32_storage == "residual" else "fp32-lean")
    t0 = time.perf_counter()
    u0 = thermalise(a.nc, a.dims, a.beta, a.dt, a.level, a.nsteps, a.therm, a.seed, **kw)
    rep = {"config": vars(a), "therm_seconds": time.perf_counter() - t0}
    rep.update(compare(a.nc, a.dims, a.beta, a.dt, a.level, a.nsteps, u0, a.dh_traj, **kw))
    if a.ensemble:
        rep["ensemble"] = ensemble(a.nc, a.dims, a.beta, a.dt, a.level, a.nsteps, u0, a.ensemble, **kw)
    print(json.dumps(rep))


if __name__ == "__main__":
    main()
