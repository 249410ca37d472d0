"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own sun.cpp / measurements4d.cpp routines (compiled
unchanged against the project's GSL shim into oracle/_ref by oracle/Makefile)
on seeded synthetic inputs and stores inputs and outputs as .npz.  Needs the
reference sources, so it runs where they are (never on the GPU host); the
committed .npz files are what the tests read.

    python tests/golden/gen_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle import Oracle, Reference, fields  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# name, NC, dims, BETA, LEVEL, start ("hot" Haar / "near" exp(i 0.3 H)), eps_E, eps_U, leapfrog steps
CASES = [
    ("su2_d2_4x5", 2, [4, 5], 2.3, 8, "hot", 0.013, 0.02, 6),
    ("su3_d4_4x3x3x2", 3, [4, 3, 3, 2], 5.7, 8, "hot", 0.01, 0.02, 5),
    ("su3_d4_3x2x1x4", 3, [3, 2, 1, 4], 6.0, 6, "hot", 0.02, 0.02, 4),
    ("su4_d3_3x3x2", 4, [3, 3, 2], 8.0, 8, "near", 0.015, 0.01, 5),
    ("su5_d3_2x3x3", 5, [2, 3, 3], 12.0, 7, "hot", 0.01, 0.01, 3),
    ("su8_d4_2x2x2x2", 8, [2, 2, 2, 2], 20.0, 8, "hot", 0.01, 0.01, 3),
    ("su3_d1_5", 3, [5], 5.7, 8, "hot", 0.02, 0.02, 3),
]


def make_case(name, nc, dims, beta, level, start, eps_e, eps_u, nlf, seed):
    rng = np.random.default_rng(seed)
    O = Oracle(nc, dims)
    R = Reference(nc, dims, beta=beta, level=level)
    R.threads(1)
    nl = O.vol * O.dim
    if start == "hot":
        u = fields.haar(nc, nl, rng).reshape(O.shape)
    else:
        u = fields.near_identity(nc, nl, 0.3, rng).reshape(O.shape)
    pi = fields.momenta(nc, nl, beta, rng, O)
    out = dict(nc=nc, dims=np.array(dims), beta=beta, level=level, eps_e=eps_e, eps_u=eps_u, u=u, pi=pi)
    # geometry
    plus = np.array([[R.getplus(s, d) for s in range(O.vol)] for d in range(O.dim)])
    minus = np.array([[R.getminus(s, d) for s in range(O.vol)] for d in range(O.dim)])
    out.update(getplus=plus, getminus=minus)
    # observables on the input configuration
    R.set("u", u)
    R.set("pi", pi)
    out["EnergyMag"] = R.EnergyMag()
    out["simpleenergyEl_pi"] = R.simpleenergyEl("pi")
    out["UViol"] = R.UViol()
    out["WilsonLoop_sun"] = R.WilsonLoop_sun()
    if O.dim >= 2:
        out["PolyakovLoop"] = R.PolyakovLoop()
        out["WilsonLoopDir"] = np.array([R.WilsonLoopDir(d) for d in range(1, O.dim)])
        out["PlaqExp"] = np.array(R.PlaqExp())
        out["scalarLoopcorr"] = R.scalarLoopcorr()
    # one force evaluation (updateE) and one link update (updateUandcopyDown)
    R.updateE(eps_e)
    out["Pi"] = R.get("Pi")
    out["simpleenergyEl_Pi"] = R.simpleenergyEl("Pi")
    out["EnergyEl"] = R.EnergyEl()
    out["GaussLaw_before"] = R.GaussLaw()
    out["TotalEnergy_before"] = R.sun.ref_TotalEnergy()
    R.updateUandcopyDown(eps_u)
    out["u_after"] = R.get("u")
    out["pi_after"] = R.get("pi")
    out["EnergyMag_after"] = R.EnergyMag()
    out["UViol_after"] = R.UViol()
    # leapfrog as sun.cpp runs it: updateE(dt/2); copyDown; [updateUandcopyDown(dt); updateE(dt)] ... ;
    # last drift followed by updateE(dt/2) -- from the same (u, pi)
    # copyDown (sun.cpp:792-801) also copies U -> u, so U must hold the start too
    R.set("u", u)
    R.set("U", u)
    R.set("pi", pi)
    dt = eps_u
    R.updateE(dt / 2)
    R.sun.ref_copyDown()
    for k in range(nlf):
        R.updateUandcopyDown(dt)
        R.updateE(dt if k < nlf - 1 else dt / 2)
    out["lf_steps"] = nlf
    out["lf_u"] = R.get("u")
    out["lf_Pi"] = R.get("Pi")
    out["lf_H_old"] = beta * (out["EnergyMag"] + out["simpleenergyEl_pi"] / (2 * nc))
    out["lf_H_new"] = beta * (R.EnergyMag() + R.simpleenergyEl("Pi") / (2 * nc))
    # matrix kernels
    m = fields.random_hermitian_traceless(nc, 1, rng)[0] * 0.7
    out["mexpi_in"] = m
    out["mexpi_out"] = np.array([R.mexpi(m, L) for L in range(0, 10)])
    a = rng.standard_normal((nc, nc)) + 1j * rng.standard_normal((nc, nc))
    out["adjoint_in"] = a
    out["adjoint_out"] = R.adjoint(a)
    out["generators"] = R.generators()
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **out)
    return out


def main():
    if not oracle.build_reference():
        raise SystemExit("reference sources not found; golden fixtures can only be regenerated next to them")
    for i, c in enumerate(CASES):
        make_case(*c, seed=1000 + i)
        print("wrote", c[0])


if __name__ == "__main__":
    main()
