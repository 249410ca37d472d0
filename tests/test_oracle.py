"""The CPU oracle (oracle/askja_oracle.c) against the reference's own routines:
the committed golden fixtures (made by tests/golden/gen_golden.py from the
reference's sun.cpp/measurements4d.cpp) and, where oracle/_ref is built, the
reference harness directly on fresh random inputs."""
import os

import numpy as np
import pytest

import oracle
from oracle import Oracle, Reference, fields
from conftest import rel

TOL = 1e-12


def test_oracle_matches_golden(golden):
    g = golden
    O = Oracle(g["nc"], g["dims"])
    u, pi = g["u"], g["pi"]
    Pi = O.updateE(u, pi, g["eps_e"])
    assert rel(Pi, g["Pi"]) < TOL
    ua = O.updateU(u, g["Pi"], g["eps_u"], g["level"])
    assert rel(ua, g["u_after"]) < TOL
    assert O.EnergyMag(u) == pytest.approx(g["EnergyMag"], rel=TOL, abs=1e-12)
    assert O.simpleenergyEl(pi) == pytest.approx(g["simpleenergyEl_pi"], rel=TOL)
    assert O.simpleenergyEl(g["Pi"]) == pytest.approx(g["simpleenergyEl_Pi"], rel=TOL)
    assert O.EnergyEl(pi, g["Pi"]) == pytest.approx(g["EnergyEl"], rel=TOL)
    # UViol and GaussLaw are rounding-level numbers (~1e-28): compare on their scale
    assert abs(O.UViol(u) - g["UViol"]) < 1e-20
    scale = float(np.sum(np.abs(g["Pi"]) ** 2))
    assert abs(O.GaussLaw(u, g["Pi"]) - g["GaussLaw_before"]) <= 1e-12 * abs(g["GaussLaw_before"]) + 1e-20 * max(scale, 1.0) ** 2
    assert O.WilsonLoop_sun(u) == pytest.approx(g["WilsonLoop_sun"], rel=1e-11, abs=1e-13)
    if O.dim >= 2:
        assert O.PolyakovLoop(u) == pytest.approx(g["PolyakovLoop"], rel=1e-11, abs=1e-13)
        w = [O.WilsonLoopDir(u, d) for d in range(1, O.dim)]
        np.testing.assert_allclose(w, g["WilsonLoopDir"], rtol=1e-11, atol=1e-13)
        np.testing.assert_allclose(O.PlaqExp(u), g["PlaqExp"], rtol=TOL, atol=1e-12)
        np.testing.assert_allclose(O.scalarLoopcorr(u), g["scalarLoopcorr"], rtol=TOL, atol=1e-14)
    np.testing.assert_allclose(O.generators(), g["generators"], atol=1e-15)
    for L in range(10):
        assert rel(O.mexpi(g["mexpi_in"], L), g["mexpi_out"][L]) < 1e-14
    assert rel(O.adjoint(g["adjoint_in"]), g["adjoint_out"]) < 1e-15
    for d in range(O.dim):
        for s in range(O.vol):
            assert O.getplus(s, d) == g["getplus"][d, s]
            assert O.getminus(s, d) == g["getminus"][d, s]


def test_oracle_leapfrog_matches_golden(golden):
    g = golden
    O = Oracle(g["nc"], g["dims"])
    dt, n = g["eps_u"], g["lf_steps"]
    u, p = g["u"], O.updateE(g["u"], g["pi"], dt / 2)
    for k in range(n):
        u = O.updateU(u, p, dt, g["level"])
        p = O.updateE(u, p, dt if k < n - 1 else dt / 2)
    assert rel(u, g["lf_u"]) < 1e-11
    assert rel(p, g["lf_Pi"]) < 1e-11
    h_new = g["beta"] * (O.EnergyMag(u) + O.simpleenergyEl(p) / (2 * g["nc"]))
    assert h_new == pytest.approx(float(g["lf_H_new"]), rel=1e-12)


def test_generators_orthonormal():
    for nc in (2, 3, 4, 5, 8):
        T = Oracle(nc, [2]).generators()
        gram = np.einsum("aij,bji->ab", T, T)
        np.testing.assert_allclose(gram, 0.5 * np.eye(nc * nc - 1), atol=1e-14)
        for t in T:
            np.testing.assert_allclose(t, t.conj().T, atol=0)
            assert abs(np.trace(t)) < 1e-14


def test_cold_start_known_answers():
    O = Oracle(3, [3, 2, 2, 4])
    u = np.zeros(O.shape, np.complex128)
    u[..., :, :] = np.eye(3)
    assert O.EnergyMag(u) == 0.0
    assert O.UViol(u) == 0.0
    assert O.PolyakovLoop(u) == pytest.approx(1.0)
    assert O.WilsonLoop_sun(u) == pytest.approx(1.0)
    p = np.zeros(O.shape, np.complex128)
    np.testing.assert_array_equal(O.updateE(u, p, 0.1), 0)


def test_momentum_normalisation():
    """P = sqrt(2N/beta) sum xi_a T_a  =>  sum tr2(P) = (N/beta) sum xi^2."""
    O = Oracle(4, [2, 3])
    xi = np.random.default_rng(3).standard_normal(O.vol * O.dim * 15)
    p = O.momenta_from_normals(xi, 7.0)
    assert O.simpleenergyEl(p) == pytest.approx(4 / 7.0 * np.sum(xi ** 2), rel=1e-13)
    np.testing.assert_allclose(p, np.conj(np.swapaxes(p, -1, -2)), atol=1e-15)


def test_philox_known_answers():
    """Philox4x32-10 known-answer vectors (Salmon et al., SC'11 / Random123)."""
    import ctypes
    O = Oracle(2, [2])
    cases = [
        ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
         (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
    ]
    for ctr, key, want in cases:
        c = (ctypes.c_uint32 * 4)(*ctr)
        k = (ctypes.c_uint32 * 2)(*key)
        o = (ctypes.c_uint32 * 4)()
        O.lib.or_philox4x32_10(c, k, o)
        assert tuple(o) == want


def test_engine_normals_statistics():
    O = Oracle(3, [8, 8, 8])
    xi = O.engine_normals(seed=42, traj=0)
    assert abs(xi.mean()) < 0.02 and abs(xi.var() - 1) < 0.03
    assert not np.array_equal(xi, O.engine_normals(seed=42, traj=1))


def test_reunitarise_projects_to_su_n():
    rng = np.random.default_rng(5)
    for nc in (2, 3, 4, 6):
        O = Oracle(nc, [3])
        u = fields.haar(nc, 10, rng)
        noisy = u + 1e-4 * (rng.standard_normal(u.shape) + 1j * rng.standard_normal(u.shape))
        r = O.reunitarise(noisy)
        eye = np.eye(nc)
        np.testing.assert_allclose(np.einsum("lij,lkj->lik", r, r.conj()), np.broadcast_to(eye, r.shape), atol=1e-13)
        np.testing.assert_allclose(np.linalg.det(r), 1.0, atol=1e-13)
        assert np.abs(r - u).max() < 1e-3
        # an exact SU(N) matrix is a fixed point
        np.testing.assert_allclose(O.reunitarise(u), u, atol=1e-13)


@pytest.mark.skipif(not Reference.available(), reason="oracle/_ref not built (needs the reference sources)")
@pytest.mark.parametrize("nc,dims", [(2, [3, 4]), (3, [2, 3, 2, 3]), (4, [1, 3, 3]), (6, [2, 2, 3]), (3, [4, 1, 1, 2])])
def test_oracle_matches_reference_random(nc, dims):
    rng = np.random.default_rng(nc * 100 + len(dims))
    O = Oracle(nc, dims)
    R = Reference(nc, dims, beta=3.0, level=7)
    nl = O.vol * O.dim
    u = fields.haar(nc, nl, rng).reshape(O.shape)
    pi = fields.momenta(nc, nl, 3.0, rng, O)
    R.set("u", u)
    R.set("pi", pi)
    R.updateE(0.03)
    assert rel(O.updateE(u, pi, 0.03), R.get("Pi")) < 1e-12
    R.updateUandcopyDown(0.05)
    assert rel(O.updateU(u, O.updateE(u, pi, 0.03), 0.05, 7), R.get("u")) < 1e-12
    R.set("u", u)
    assert O.EnergyMag(u) == pytest.approx(R.EnergyMag(), rel=1e-12)


def test_ensemble_fixture_consistent():
    """The reference-run ensemble fixture (tests/golden/gen_ensemble.py): its
    binned series reproduce the Nrav averages the reference's measure4d wrote
    (printed to 6 digits), and the run kept every trajectory's configuration."""
    import json
    fx = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                     "ensemble_su3_4x4x4x4.json")))
    assert fx["taken"] == fx["params"]["trajectories"]
    n = fx["taken"] - fx["skip"]
    for k in ("polyakov", "wilson", "plaq_t", "plaq_s"):
        b = np.asarray(fx["bins"][k])
        assert len(b) == n // fx["bin"]
        if len(b) * fx["bin"] == n:
            assert b.mean() == pytest.approx(fx["nrav"][k], rel=1e-5)
        assert fx["nrav"][k + "_err"] > 0
