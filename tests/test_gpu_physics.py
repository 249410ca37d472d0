"""Physics properties of the GPU engine that hold at any size: cold-start
known answers, gauge invariance, reversibility, dH ~ dt^2, unitarity of the
hot start and of the FP32 path, momentum statistics, graph replay ==
eager, accept/reject bookkeeping, NaN rejection."""
import numpy as np
import pytest

import askja_b200 as ab
from oracle import Oracle, fields
from conftest import rel

pytestmark = pytest.mark.gpu


def gauge_transform(u, dims, g):
    """U_mu(x) -> g(x) U_mu(x) g(x+mu)^dag."""
    V, D = u.shape[:2]
    O = Oracle(u.shape[-1], dims)
    out = np.empty_like(u)
    for mu in range(D):
        plus = np.array([O.getplus(s, mu) for s in range(V)])
        out[:, mu] = np.einsum("sij,sjk,slk->sil", g, u[:, mu], g[plus].conj())
    return out


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_cold_start(precision):
    with ab.Engine(3, [4, 4, 4, 4], beta=5.7, precision=precision) as e:
        e.initializeU()
        assert e.EnergyMag() == 0.0
        assert e.PlaqExp() == (0.0, 0.0)
        assert e.UViol() == 0.0
        assert e.PolyakovLoop() == pytest.approx(1.0, abs=1e-15)
        assert e.WilsonLoop() == pytest.approx(1.0, abs=1e-15)
        e.set_momenta(np.zeros(e.shape), 0)
        e.updateE(0.1)
        assert np.abs(e.get_momenta(1)).max() == 0.0


@pytest.mark.parametrize("nc", [2, 3, 5])
def test_gauge_invariance(nc):
    dims = [3, 4, 2, 3]
    rng = np.random.default_rng(nc)
    O = Oracle(nc, dims)
    u = fields.haar(nc, O.vol * O.dim, rng).reshape(O.shape)
    g = fields.haar(nc, O.vol, rng)
    ug = gauge_transform(u, dims, g)
    with ab.Engine(nc, dims, beta=4.0) as e:
        e.set_links(u)
        s0, p0, pl0 = e.EnergyMag(), e.PlaqExp(), e.PolyakovLoop()
        e.set_links(ug)
        assert e.EnergyMag() == pytest.approx(s0, rel=1e-12)
        np.testing.assert_allclose(e.PlaqExp(), p0, rtol=1e-12)
        assert e.PolyakovLoop() == pytest.approx(pl0, rel=1e-11)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("fp32", 5e-5)])
def test_reversibility(precision, tol):
    """Integrate forward, flip P, integrate back: back at U_0 (no reunitarisation)."""
    nc, dims = 3, [4, 4, 4, 4]
    rng = np.random.default_rng(7)
    O = Oracle(nc, dims)
    u0 = fields.near_identity(nc, O.vol * O.dim, 0.5, rng).reshape(O.shape)
    p0 = fields.momenta(nc, O.vol * O.dim, 5.7, rng, O)
    with ab.Engine(nc, dims, beta=5.7, level=8, precision=precision, reunitarise=False) as e:
        e.set_links(u0)
        e.set_momenta(p0, 0)
        e.leapfrog(10, 0.02)
        p1 = e.get_momenta(0)
        e.set_momenta(-p1, 0)
        e.leapfrog(10, 0.02)
        assert np.abs(e.get_links() - u0).max() < tol
        assert rel(-e.get_momenta(0), p0) < 10 * tol


def test_dh_scales_as_dt_squared():
    nc, dims, beta = 3, [4, 4, 4, 4], 5.7
    rng = np.random.default_rng(9)
    O = Oracle(nc, dims)
    u0 = fields.near_identity(nc, O.vol * O.dim, 0.6, rng).reshape(O.shape)
    p0 = fields.momenta(nc, O.vol * O.dim, beta, rng, O)
    dhs = []
    for dt in (0.04, 0.02, 0.01):
        with ab.Engine(nc, dims, beta=beta, level=8) as e:
            e.set_links(u0)
            e.set_momenta(p0, 0)
            h0 = e.hamiltonian(0)
            e.leapfrog(int(round(0.4 / dt)), dt)
            dhs.append(abs(e.hamiltonian(0) - h0))
    assert 2.5 < dhs[0] / dhs[1] < 6 and 2.5 < dhs[1] / dhs[2] < 6


@pytest.mark.parametrize("nc", [2, 3, 4, 6, 8])
def test_hot_start_is_su_n(nc):
    with ab.Engine(nc, [8, 8, 4], beta=1.0) as e:
        e.hot_start(1234)
        u = e.get_links().reshape(-1, nc, nc)
        eye = np.eye(nc)
        assert np.abs(np.einsum("lij,lkj->lik", u, u.conj()) - eye).max() < 1e-13
        np.testing.assert_allclose(np.linalg.det(u), 1.0, atol=1e-13)
        # Haar: <|Tr U|^2> = 1 for SU(N), N >= 2
        assert abs(np.mean(np.abs(np.trace(u, axis1=1, axis2=2)) ** 2) - 1.0) < 0.15
        np.testing.assert_array_equal(e.get_saved_links().reshape(-1, nc, nc), u)


def test_fp32_reunitarised_trajectories_stay_unitary():
    with ab.Engine(3, [8, 8, 8, 8], beta=5.7, dt=0.02, level=6, precision="fp32", seed=5) as e:
        e.hot_start(77)
        e.run_trajectories(3, 20, use_graph=True)
        assert e.UViol() / (e.vol * e.dim) < 1e-12


@pytest.mark.parametrize("nc", [3, 8, 16, 32])
def test_momentum_refresh_matches_oracle(nc):
    """Thread-per-link refresh (NC < 16) and CTA-per-link refresh (NC >= 16)."""
    dims, beta, seed = ([4, 3, 2, 2] if nc < 32 else [2, 3, 2]), 4.5, 31337
    O = Oracle(nc, dims)
    with ab.Engine(nc, dims, beta=beta) as e:
        e.initializeE(seed, 5)
        want = O.momenta_from_normals(O.engine_normals(seed, 5), beta)
        assert rel(e.get_momenta(0), want) < 1e-13


def test_momentum_statistics():
    nc, beta = 3, 6.0
    with ab.Engine(nc, [8, 8, 8, 8], beta=beta) as e:
        e.initializeE(1, 0)
        k = e.simpleenergyEl(0)
        # <sum tr2 P> = (N/beta) * (N^2-1) * links
        expect = nc / beta * (nc * nc - 1) * e.vol * e.dim
        assert k == pytest.approx(expect, rel=0.01)
        p = e.get_momenta(0).reshape(-1, nc, nc)
        np.testing.assert_allclose(p, np.conj(np.swapaxes(p, 1, 2)), atol=1e-15)
        assert np.abs(np.trace(p, axis1=1, axis2=2)).max() < 1e-14


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_graph_replay_equals_eager(precision):
    args = dict(nc=3, dims=[4, 4, 4, 4], beta=5.7, dt=0.02, level=8, precision=precision, seed=99)
    res = []
    for use_graph in (False, True):
        with ab.Engine(**args) as e:
            e.hot_start(3)
            last, log = e.run_trajectories(4, 7, use_graph=use_graph)
            res.append((last, log, e.get_links()))
    assert res[0][0] == res[1][0]
    np.testing.assert_array_equal(res[0][1], res[1][1])
    np.testing.assert_array_equal(res[0][2], res[1][2])


def test_acceptance_bookkeeping():
    with ab.Engine(3, [4, 4, 4, 4], beta=5.7, dt=0.02, level=8, seed=4) as e:
        e.hot_start(8)
        last, log = e.run_trajectories(6, 10, use_graph=True)
        assert last["n_tot"] == 6 == last["n_acc"] + last["n_rej"]
        assert last["n_acc1"] == int(np.sum(log[:, 3] == 1))
        assert last["n_acc"] == int(np.sum(log[:, 3] > 0))
        np.testing.assert_allclose(log[:, 2], log[:, 1] - log[:, 0], atol=1e-9)
        assert np.all(np.isfinite(log))


def test_reject_restores_configuration():
    """A huge dt makes dH enormous (or overflows the Taylor series to NaN, which
    fails both acceptance tests exactly as in the reference): the trajectory is
    rejected and u = uconf = start."""
    with ab.Engine(3, [4, 4, 2, 2], beta=5.7, dt=1.5, level=8, seed=4) as e:
        e.hot_start(8)
        u0 = e.get_links()
        r = e.trajectory(3)
        assert r["accepted"] == 0 and (np.isnan(r["dh"]) or r["dh"] > 50)
        np.testing.assert_array_equal(e.get_links(), u0)
        np.testing.assert_array_equal(e.get_saved_links(), u0)


def test_nonfinite_upload_rejected():
    with ab.Engine(2, [4, 4], beta=2.0) as e:
        e.initializeU()
        u = e.get_links()
        bad = u.copy()
        bad[3, 1, 0, 1] = np.nan
        with pytest.raises(ab.AskjaError) as ex:
            e.set_links(bad)
        assert ex.value.code == -4
        np.testing.assert_array_equal(e.get_links(), u)


def test_invalid_arguments():
    with pytest.raises(ab.AskjaError) as ex:
        ab.Engine(1, [4, 4], beta=1.0)
    assert ex.value.code == -1
    with pytest.raises(ab.AskjaError):
        ab.Engine(3, [4, 0], beta=1.0)
    with ab.Engine(3, [4, 4], beta=1.0) as e:
        with pytest.raises(ab.AskjaError):
            e.WilsonLoopDir(0)
        with pytest.raises(ab.AskjaError):
            e.trajectory(0)


def test_precision_module_small():
    """askja_b200.precision on a small lattice: FP32-mixed stays within
    FP32-level distance of FP64 on identical inputs."""
    from askja_b200 import precision
    nc, dims, beta, dt, level, n = 3, [6, 6, 6, 6], 5.7, 0.02, 8, 10
    u0 = precision.thermalise(nc, dims, beta, dt, level, n, 5, 3)
    r = precision.compare(nc, dims, beta, dt, level, n, u0, ntraj_dh=2)
    assert r["force_rel_err"] < 2e-5
    assert r["max_abs_dH_diff"] < 5e-3
    assert r["reversibility"]["fp64"] < 1e-10 and r["reversibility"]["fp32"] < 1e-5
    assert r["unitarity_max"] < 5e-6
    ens = precision.ensemble(nc, dims, beta, dt, level, n, u0, 10)
    # a few trajectories from a hot start: far from equilibrium, but moving up from 0
    assert 0.05 < ens["fp64"]["plaquette"] < 0.8 and 0.05 < ens["fp32"]["plaquette"] < 0.8
    # temporal and spatial planes average to the whole (3 of each in D = 4)
    for k in ("fp64", "fp32"):
        e = ens[k]
        assert e["plaquette"] == pytest.approx(0.5 * (e["plaquette_t"] + e["plaquette_s"]), rel=1e-12)
        assert abs(e["wilson"]) <= 1.0 + 1e-12
    assert abs(ens["plaquette_t_diff"]) < 0.05 and abs(ens["wilson_diff"]) < 0.5
