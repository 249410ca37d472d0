"""GPU engine (through the C ABI) against the reference's own outputs (golden
fixtures from tests/golden/gen_golden.py) and against the FP64 CPU oracle.

Tolerances: the FP64 path must agree to relative 1e-12 on force, one link
update, action, kinetic sums and one leapfrog trajectory (it is not bit-exact:
reduction order and the factoring of the staple product differ).  The FP32
path is checked against the same FP64 answers with FP32-level tolerances
(relative 2e-5 on fields, 1e-6 relative on the FP64-accumulated sums)."""
import os

import numpy as np
import pytest

import askja_b200 as ab
from conftest import rel
from oracle import Oracle, Reference, fields

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def engine_for(g, precision="fp64", kernel_path=0, reunit=None):
    return ab.Engine(g["nc"], g["dims"], beta=g["beta"], dt=g["eps_u"], level=g["level"], precision=precision,
                     kernel_path=kernel_path, reunitarise=reunit)


@pytest.mark.parametrize("kernel_path", [0, 1])
def test_fp64_matches_golden(golden, kernel_path):
    g = golden
    with engine_for(g, kernel_path=kernel_path) as e:
        e.set_links(g["u"])
        e.set_momenta(g["pi"], 0)
        np.testing.assert_array_equal(e.get_links(), g["u"])
        assert e.EnergyMag() == pytest.approx(g["EnergyMag"], rel=TOL64, abs=1e-12)
        assert e.simpleenergyEl(0) == pytest.approx(g["simpleenergyEl_pi"], rel=TOL64)
        assert abs(e.UViol() - g["UViol"]) < 1e-20
        assert e.WilsonLoop() == pytest.approx(g["WilsonLoop_sun"], rel=1e-11, abs=1e-13)
        if e.dim >= 2:
            assert e.PolyakovLoop() == pytest.approx(g["PolyakovLoop"], rel=1e-11, abs=1e-13)
            w = [e.WilsonLoopDir(d) for d in range(1, e.dim)]
            np.testing.assert_allclose(w, g["WilsonLoopDir"], rtol=1e-11, atol=1e-13)
            np.testing.assert_allclose(e.PlaqExp(), g["PlaqExp"], rtol=TOL64, atol=1e-12)
            np.testing.assert_allclose(e.scalarLoopcorr(), g["scalarLoopcorr"], rtol=TOL64, atol=1e-14)
        e.updateE(g["eps_e"])
        assert rel(e.get_momenta(1), g["Pi"]) < TOL64
        assert e.simpleenergyEl(1) == pytest.approx(g["simpleenergyEl_Pi"], rel=TOL64)
        assert e.EnergyEl() == pytest.approx(g["EnergyEl"], rel=TOL64)
        scale = float(np.sum(np.abs(g["Pi"]) ** 2))
        assert abs(e.GaussLaw() - g["GaussLaw_before"]) <= 1e-12 * abs(g["GaussLaw_before"]) + 1e-20 * max(scale, 1.0) ** 2
        assert e.TotalEnergy() == pytest.approx(g["TotalEnergy_before"], rel=TOL64)
        e.updateUandcopyDown(g["eps_u"])
        assert rel(e.get_links(), g["u_after"]) < TOL64
        assert rel(e.get_momenta(0), g["pi_after"]) < TOL64
        assert e.EnergyMag() == pytest.approx(g["EnergyMag_after"], rel=TOL64, abs=1e-12)


@pytest.mark.parametrize("kernel_path", [0, 1])
def test_fp64_leapfrog_matches_golden(golden, kernel_path):
    """One leapfrog trajectory, reference step order, fused kernels."""
    g = golden
    with engine_for(g, kernel_path=kernel_path) as e:
        e.set_links(g["u"])
        e.set_momenta(g["pi"], 0)
        e.leapfrog(g["lf_steps"], g["eps_u"])
        assert rel(e.get_links(), g["lf_u"]) < TOL64
        assert rel(e.get_momenta(0), g["lf_Pi"]) < TOL64
        h_new = e.hamiltonian(0)
        assert h_new == pytest.approx(float(g["lf_H_new"]), rel=TOL64)


def test_fp64_md_steps_match_seam(golden):
    """askja_md_steps (fused) == n x (updateUandcopyDown; updateE), pi and Pi both."""
    g = golden
    with engine_for(g) as a, engine_for(g) as b:
        for e in (a, b):
            e.set_links(g["u"])
            e.set_momenta(g["pi"], 0)
            e.updateE(0.5 * g["eps_u"])
        a.md_steps(3, g["eps_u"])
        for _ in range(3):
            b.updateUandcopyDown(g["eps_u"])
            b.updateE(g["eps_u"])
        assert rel(a.get_links(), b.get_links()) < 1e-13
        assert rel(a.get_momenta(0), b.get_momenta(0)) < 1e-13
        assert rel(a.get_momenta(1), b.get_momenta(1)) < 1e-13


def test_fp32_matches_golden(golden):
    g = golden
    with engine_for(g, precision="fp32", reunit=False) as e:
        e.set_links(g["u"])
        e.set_momenta(g["pi"], 0)
        assert e.EnergyMag() == pytest.approx(g["EnergyMag"], rel=2e-6, abs=1e-5)
        e.updateE(g["eps_e"])
        assert rel(e.get_momenta(1), g["Pi"]) < 2e-5
        e.updateUandcopyDown(g["eps_u"])
        assert rel(e.get_links(), g["u_after"]) < 2e-6
        e.set_links(g["u"])
        e.set_momenta(g["pi"], 0)
        e.leapfrog(g["lf_steps"], g["eps_u"])
        assert rel(e.get_links(), g["lf_u"]) < 2e-5
        assert e.hamiltonian(0) == pytest.approx(float(g["lf_H_new"]), rel=2e-6)


CASES = [(2, [6, 4, 3, 5]), (3, [4, 4, 4, 4]), (3, [5, 1, 2, 3]), (4, [3, 4, 5]), (5, [3, 3, 2, 2]),
         (6, [2, 3, 4]), (8, [3, 3, 2, 2]), (9, [2, 2, 3]), (12, [2, 2, 2]), (16, [2, 3]),
         (3, [7]), (5, [4])]  # DIM 1: no plaquettes, zero force


@pytest.mark.parametrize("nc,dims", CASES, ids=[f"su{n}_{'x'.join(map(str, d))}" for n, d in CASES])
def test_fp64_force_link_action_vs_oracle(nc, dims):
    rng = np.random.default_rng(nc * 7 + len(dims))
    O = Oracle(nc, dims)
    nl = O.vol * O.dim
    u = fields.haar(nc, nl, rng).reshape(O.shape)
    beta = 2.0 * nc
    pi = fields.momenta(nc, nl, beta, rng, O)
    with ab.Engine(nc, dims, beta=beta, dt=0.02, level=8) as e:
        e.set_links(u)
        e.set_momenta(pi, 0)
        e.updateE(0.02)
        Pi = O.updateE(u, pi, 0.02)
        assert rel(e.get_momenta(1), Pi) < TOL64
        e.updateUandcopyDown(0.03)
        ua = O.updateU(u, Pi, 0.03, 8)
        assert rel(e.get_links(), ua) < TOL64
        assert e.EnergyMag() == pytest.approx(O.EnergyMag(ua), rel=TOL64)
        assert e.simpleenergyEl(0) == pytest.approx(O.simpleenergyEl(Pi), rel=TOL64)
        if len(dims) >= 2:
            assert e.PolyakovLoop() == pytest.approx(O.PolyakovLoop(ua), rel=1e-11)


@pytest.mark.parametrize("level", [0, 1, 2, 5, 8, 9, -3])
def test_taylor_levels(level):
    """LEVEL semantics of mexpi: 0..8 as given, anything else = 8 (sunmat.h:215-246)."""
    nc, dims = 3, [3, 2, 2]
    rng = np.random.default_rng(11)
    O = Oracle(nc, dims)
    u = fields.haar(nc, O.vol * O.dim, rng).reshape(O.shape)
    Pi = fields.momenta(nc, O.vol * O.dim, 1.0, rng, O)
    with ab.Engine(nc, dims, beta=1.0, level=level) as e:
        e.set_links(u)
        e.set_momenta(Pi, 1)
        e.updateUandcopyDown(0.1)
        assert rel(e.get_links(), O.updateU(u, Pi, 0.1, level)) < TOL64


def test_trajectory_matches_oracle():
    """askja_trajectory: Philox momenta, leapfrog, H_old/H_new and Metropolis,
    reproduced step by step with the oracle."""
    nc, dims, beta, dt, n = 3, [4, 3, 3, 2], 5.7, 0.02, 6
    rng = np.random.default_rng(21)
    O = Oracle(nc, dims)
    u = fields.haar(nc, O.vol * O.dim, rng).reshape(O.shape)
    seed = 987654321
    with ab.Engine(nc, dims, beta=beta, dt=dt, level=8, seed=seed) as e:
        e.set_links(u)
        r = e.trajectory(n)
        xi = O.engine_normals(seed, 0)
        p = O.momenta_from_normals(xi, beta)
        h_old = beta * (O.EnergyMag(u) + O.simpleenergyEl(p) / (2 * nc))
        uu, pp = u, O.updateE(u, p, dt / 2)
        for k in range(n):
            uu = O.updateU(uu, pp, dt, 8)
            pp = O.updateE(uu, pp, dt if k < n - 1 else dt / 2)
        h_new = beta * (O.EnergyMag(uu) + O.simpleenergyEl(pp) / (2 * nc))
        assert r["h_old"] == pytest.approx(h_old, rel=1e-12)
        assert r["h_new"] == pytest.approx(h_new, rel=1e-12)
        assert r["dh"] == pytest.approx(h_new - h_old, abs=1e-9)
        acc = r["accepted"] != 0
        assert r["n_tot"] == 1 and r["traj"] == 1
        assert rel(e.get_saved_links(), uu if acc else u) < 1e-12
        assert rel(e.get_links(), uu if acc else u) < 1e-12


@pytest.mark.parametrize("nc,dims,precision", [(24, [2, 2, 2], "fp64"), (32, [2, 2, 2], "fp64"), (64, [2, 2], "fp64"),
                                               (32, [2, 2, 2], "fp32"), (64, [2, 2], "fp32")])
def test_large_nc_vs_oracle(nc, dims, precision):
    """Large colour numbers (config 5's SU(32)/SU(64)) on tiny lattices."""
    rng = np.random.default_rng(nc)
    O = Oracle(nc, dims)
    nl = O.vol * O.dim
    u = fields.haar(nc, nl, rng).reshape(O.shape)
    beta = 2.0 * nc * nc
    pi = fields.momenta(nc, nl, beta, rng, O)
    tol = TOL64 if precision == "fp64" else 5e-5
    with ab.Engine(nc, dims, beta=beta, dt=0.005, level=8, precision=precision, reunitarise=False) as e:
        e.set_links(u)
        e.set_momenta(pi, 0)
        e.updateE(0.005)
        Pi = O.updateE(u, pi, 0.005)
        assert rel(e.get_momenta(1), Pi) < tol
        e.updateUandcopyDown(0.005)
        assert rel(e.get_links(), O.updateU(u, Pi, 0.005, 8)) < (TOL64 if precision == "fp64" else 5e-6)
        e.set_links(u)
        e.set_momenta(pi, 0)
        e.leapfrog(2, 0.005)
        uu, pp = u, O.updateE(u, pi, 0.0025)
        for k in range(2):
            uu = O.updateU(uu, pp, 0.005, 8)
            pp = O.updateE(uu, pp, 0.005 if k < 1 else 0.0025)
        assert rel(e.get_links(), uu) < (TOL64 if precision == "fp64" else 5e-6)


@pytest.mark.skipif(not Reference.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("start", ["cold", "hot"])
def test_config1_step_by_step_vs_reference(start):
    """SU(3) 8^4, BETA=5.70, DT=0.02, LEVEL=8, 50 leapfrog steps: the FP64
    engine and the reference's own sun.cpp routines (the shim-built harness)
    take the same U and P and the same updateE / updateUandcopyDown sequence
    (sun.cpp:1174-1250); links, momenta and H agree after every step.  The
    Metropolis decision itself uses each side's own random stream."""
    nc, dims, beta, dt, level, nsteps = 3, [8, 8, 8, 8], 5.70, 0.02, 8, 50
    rng = np.random.default_rng(1 if start == "cold" else 2)
    O = Oracle(nc, dims)
    nl = O.vol * O.dim
    if start == "cold":
        u = np.broadcast_to(np.eye(nc, dtype=np.complex128), O.shape).copy()
    else:
        u = fields.haar(nc, nl, rng).reshape(O.shape)
    pi = fields.momenta(nc, nl, beta, rng, O)
    R = Reference(nc, dims, beta=beta, level=level)
    R.threads(os.cpu_count() or 1)
    for name in ("u", "U"):
        R.set(name, u)
    R.set("pi", pi)
    R.set("Pi", pi)

    def ham(emag, k):
        return beta * (emag + k / (2 * nc))

    with ab.Engine(nc, dims, beta=beta, dt=dt, level=level) as e:
        e.set_links(u)
        e.set_momenta(pi, 0)
        h0_ref = ham(R.EnergyMag(), R.simpleenergyEl("pi"))
        assert e.hamiltonian(0) == pytest.approx(h0_ref, rel=1e-13)
        R.updateE(0.5 * dt)
        e.updateE(0.5 * dt)
        for k in range(nsteps):
            R.updateUandcopyDown(dt)
            e.updateUandcopyDown(dt)
            last = k == nsteps - 1
            R.updateE(0.5 * dt if last else dt)
            e.updateE(0.5 * dt if last else dt)
            assert rel(e.get_links(), R.get("u")) < 1e-11, k
            assert rel(e.get_momenta(1), R.get("Pi")) < 1e-11, k
        h1_ref = ham(R.EnergyMag(), R.simpleenergyEl("Pi"))
        h1 = beta * (e.EnergyMag() + e.simpleenergyEl(1) / (2 * nc))
        assert h1 == pytest.approx(h1_ref, rel=1e-12)
        assert abs((h1 - h0_ref) - (h1_ref - h0_ref)) < 1e-8
        t, s = e.PlaqExp()
        assert t + s == pytest.approx(R.EnergyMag(), rel=1e-12)


@pytest.mark.skipif(not Reference.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("precision,tol_p,tol_u", [("fp64", 1e-12, 1e-12), ("fp32", 5e-5, 5e-6)])
def test_config2_full_size_step_vs_reference(precision, tol_p, tol_u):
    """SU(8) 10^4 (40,000 links), BETA 20, DT 0.01, LEVEL 8 at full size: one
    updateE and one updateUandcopyDown of the engine against the reference's
    own sun.cpp routines (shim-built harness) on the same Haar links and
    momenta, and the action after the step."""
    nc, dims, beta, dt, level = 8, [10, 10, 10, 10], 20.0, 0.01, 8
    rng = np.random.default_rng(808)
    O = Oracle(nc, dims)
    nl = O.vol * O.dim
    u = fields.haar(nc, nl, rng).reshape(O.shape)
    pi = fields.momenta(nc, nl, beta, rng, O)
    R = Reference(nc, dims, beta=beta, level=level)
    R.threads(os.cpu_count() or 1)
    for name in ("u", "U"):
        R.set(name, u)
    R.set("pi", pi)
    R.set("Pi", pi)
    R.updateE(dt)
    with ab.Engine(nc, dims, beta=beta, dt=dt, level=level, precision=precision, reunitarise=False) as e:
        e.set_links(u)
        e.set_momenta(pi, 0)
        assert e.EnergyMag() == pytest.approx(O.EnergyMag(u), rel=1e-12 if precision == "fp64" else 1e-6)
        e.updateE(dt)
        assert rel(e.get_momenta(1), R.get("Pi")) < tol_p
        R.updateUandcopyDown(dt)
        e.updateUandcopyDown(dt)
        assert rel(e.get_links(), R.get("u")) < tol_u
        assert rel(e.get_momenta(0), R.get("pi")) < tol_p
        assert e.EnergyMag() == pytest.approx(R.EnergyMag(), rel=1e-12 if precision == "fp64" else 1e-6)
