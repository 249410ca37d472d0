"""The residual-plane FP32 mode (ASKJA_FP32, NC <= 4): FP32 arithmetic on
fields that carry bfloat16 residuals, against the FP64 oracle and the FP64
engine.

Tolerances.  hi + lo holds a value to ~2^-33 relative, so uploads round-trip
to 1e-10 and the FP64 reductions agree with the oracle to 1e-9.  The force
and the exponential are computed in FP32 from the FP32 part, so fields after a
few MD steps differ from FP64 by ~1e-8 relative (the FP32-only storage:
~1e-6).  The point of the mode is the energy: |dH32 - dH64| per trajectory on
a thermalised SU(3) 8^4 lattice stays at the 1e-5 level (FP32-only storage:
1e-4 to 6e-4, growing as the square root of the volume)."""
import numpy as np
import pytest

import askja_b200 as ab
from conftest import rel
from oracle import Oracle, fields

pytestmark = pytest.mark.gpu

CASES = [(2, [6, 4, 3, 5]), (3, [4, 4, 4, 4]), (3, [5, 1, 2, 3]), (4, [3, 4, 5]), (3, [7])]
IDS = [f"su{n}_{'x'.join(map(str, d))}" for n, d in CASES]


def setup(nc, dims, seed, beta=None):
    rng = np.random.default_rng(seed)
    O = Oracle(nc, dims)
    nl = O.vol * O.dim
    beta = 2.0 * nc if beta is None else beta
    return O, fields.haar(nc, nl, rng).reshape(O.shape), fields.momenta(nc, nl, beta, rng, O), beta


def oracle_leapfrog(O, u, p, n, eps, level):
    p = O.updateE(u, p, 0.5 * eps)
    for i in range(n):
        u = O.updateU(u, p, eps, level)
        p = O.updateE(u, p, eps if i < n - 1 else 0.5 * eps)
    return u, p


@pytest.mark.parametrize("nc,dims", CASES, ids=IDS)
def test_upload_and_reductions_exact(nc, dims):
    O, u, pi, beta = setup(nc, dims, 3 * nc + len(dims))
    with ab.Engine(nc, dims, beta=beta, precision="fp32") as e:
        e.set_links(u)
        e.set_momenta(pi, 0)
        assert np.abs(e.get_links() - u).max() < 1e-10
        assert np.abs(e.get_saved_links() - u).max() < 1e-10
        assert rel(e.get_momenta(0), pi) < 1e-9
        assert e.EnergyMag() == pytest.approx(O.EnergyMag(u), rel=1e-9, abs=1e-9)
        assert e.simpleenergyEl(0) == pytest.approx(O.simpleenergyEl(pi), rel=1e-9)
        assert e.UViol() / (O.vol * O.dim) < 1e-16


@pytest.mark.parametrize("nc,dims", CASES, ids=IDS)
def test_leapfrog_vs_oracle(nc, dims):
    """Four fused kick+drift steps: ~1e-8 of the FP64 answer (FP32-only: ~1e-6)."""
    O, u, pi, beta = setup(nc, dims, 5 * nc + len(dims))
    eps, level, n = 0.02, 6, 4
    want_u, want_p = oracle_leapfrog(O, u, pi, n, eps, level)
    with ab.Engine(nc, dims, beta=beta, dt=eps, level=level, precision="fp32") as e:
        e.set_links(u)
        e.set_momenta(pi, 0)
        e.leapfrog(n, eps)
        assert rel(e.get_links(), want_u) < 1e-7
        assert rel(e.get_momenta(0), want_p) < 3e-7
        assert e.hamiltonian(0) == pytest.approx(beta * (O.EnergyMag(want_u) + O.simpleenergyEl(want_p) / (2 * nc)),
                                                 rel=1e-8)


@pytest.mark.parametrize("level", [0, 1, 2, 5, 8, 9])
def test_link_update_orders(level):
    """updateE + updateUandcopyDown at every Taylor order (E - 1 formed directly)."""
    for nc in (2, 3, 4):
        dims = [3, 2, 2]
        O, u, pi, beta = setup(nc, dims, 40 + nc + level)
        with ab.Engine(nc, dims, beta=beta, level=level, precision="fp32") as e:
            e.set_links(u)
            e.set_momenta(pi, 0)
            e.updateE(0.05)
            Pi = O.updateE(u, pi, 0.05)
            assert rel(e.get_momenta(1), Pi) < 1e-7
            e.updateUandcopyDown(0.05)
            assert rel(e.get_links(), O.updateU(u, Pi, 0.05, level)) < 2e-8
            assert rel(e.get_momenta(0), Pi) < 1e-7


def test_refresh_matches_fp64_engine():
    """Same Philox stream: the coordinates hold the FP64 momenta to ~1e-10."""
    for nc in (2, 3, 4):
        dims = [4, 3, 2, 2]
        with ab.Engine(nc, dims, beta=5.0, precision="fp64") as a, \
                ab.Engine(nc, dims, beta=5.0, precision="fp32") as b:
            a.initializeE(99, 4)
            b.initializeE(99, 4)
            assert rel(b.get_momenta(0), a.get_momenta(0)) < 1e-9
            assert b.simpleenergyEl(0) == pytest.approx(a.simpleenergyEl(0), rel=1e-9)


def test_momenta_stored_in_the_algebra():
    """An uploaded matrix is replaced by its Hermitian traceless part."""
    nc, dims = 3, [2, 2, 2]
    rng = np.random.default_rng(1)
    V = 8
    m = rng.standard_normal((V, 3, nc, nc)) + 1j * rng.standard_normal((V, 3, nc, nc))
    h = 0.5 * (m + np.conj(np.swapaxes(m, -1, -2)))
    h -= np.trace(h, axis1=-2, axis2=-1)[..., None, None] / nc * np.eye(nc)
    with ab.Engine(nc, dims, beta=5.0, precision="fp32") as e:
        e.set_momenta(m, 1)
        assert rel(e.get_momenta(1), h) < 1e-9


def test_reunitarise_projects_in_fp64():
    nc, dims = 3, [4, 4, 2]
    O, u, pi, beta = setup(nc, dims, 8)
    rng = np.random.default_rng(9)
    noisy = u + 1e-6 * (rng.standard_normal(u.shape) + 1j * rng.standard_normal(u.shape))
    with ab.Engine(nc, dims, beta=beta, precision="fp32") as e:
        e.set_links(noisy)
        e.reunitarise()
        m = e.get_links().reshape(-1, nc, nc)
    assert np.abs(np.einsum("lij,lkj->lik", m, m.conj()) - np.eye(nc)).max() < 1e-9
    np.testing.assert_allclose(np.linalg.det(m), 1.0, atol=1e-9)
    assert np.abs(m - u.reshape(-1, nc, nc)).max() < 1e-5


def test_trajectories_track_fp64_engine():
    """Whole trajectories (graph replay, per-trajectory projection, Metropolis)
    on identical starts and seeds: the same decisions, energies to ~1e-8.
    From a hot start the action falls by thousands per trajectory, so the
    FP32 force's ~1e-7 relative error moves the energies by ~1e-5 here."""
    nc, dims, beta = 3, [4, 4, 4, 4], 5.7
    with ab.Engine(nc, dims, beta=beta, dt=0.02, level=6, precision="fp64", seed=21) as e:
        e.hot_start(4)
        u0 = e.get_links()
    logs = {}
    for prec in ("fp64", "fp32"):
        with ab.Engine(nc, dims, beta=beta, dt=0.02, level=6, precision=prec, seed=21) as e:
            e.set_links(u0)
            last, log = e.run_trajectories(4, 20, use_graph=True)
            logs[prec] = log
    a, b = logs["fp64"], logs["fp32"]
    np.testing.assert_array_equal(a[:, 3], b[:, 3])
    np.testing.assert_allclose(b[:, 0], a[:, 0], rtol=2e-8)
    assert np.abs(b[:, 2] - a[:, 2]).max() < 2e-4


def test_dh_tracks_fp64_on_thermalised_lattice():
    """The precision target on a thermalised SU(3) 8^4 lattice."""
    from askja_b200 import precision
    nc, dims, beta, dt, level, n = 3, [8, 8, 8, 8], 6.0, 0.02, 6, 50
    u0 = precision.thermalise(nc, dims, beta, dt, level, n, 30, 5)
    r = precision.compare(nc, dims, beta, dt, level, n, u0, ntraj_dh=3)
    assert r["max_abs_dH_diff"] < 1e-4, r["dH"]  # FP32-only storage: 1e-4 .. 6e-4 here
    assert r["force_rel_err"] < 2e-5
    assert r["reversibility"]["fp32"] < 1e-7


def test_dh_within_target_and_unbiased_at_32x4():
    """The precision target where it is hardest: SU(3) 32^4 (4.2M links),
    every trajectory within |dH32 - dH64| <= 1e-3 and their mean near zero.
    A systematic change of the link norms grows with the volume while the
    rounding noise grows with its square root, so a bias shows here first: the
    SU(3) exponential dropping its sub-ulp terms gave a mean of +1.0e-3 (now
    +1.2e-4 +- 0.5e-4 over 20 trajectories), FP32-only storage gives 1e-2."""
    from askja_b200 import precision
    nc, dims, beta, dt, level, n = 3, [32, 32, 32, 32], 6.0, 0.02, 6, 50
    u0 = precision.thermalise(nc, dims, beta, dt, level, n, 200, 5)
    r = precision.compare(nc, dims, beta, dt, level, n, u0, ntraj_dh=6)
    d = np.array([x["dH32"] - x["dH64"] for x in r["dH"]])
    assert np.abs(d).max() < 1e-3, d
    assert abs(d.mean()) < 6e-4, d


def test_autotune_keeps_the_mapping():
    nc, dims = 3, [4, 4, 4, 4]
    O, u, pi, beta = setup(nc, dims, 12)
    with ab.Engine(nc, dims, beta=beta, precision="fp32") as e:
        e.set_links(u)
        e.set_momenta(pi, 0)
        t = ab.autotune(e, reps=2)
        assert {c["path"] for c in t["candidates"]} == {0}
        assert np.abs(e.get_links() - u).max() < 1e-10
        e.leapfrog(2, 0.02)
        want_u, _ = oracle_leapfrog(O, u, pi, 2, 0.02, 8)
        assert rel(e.get_links(), want_u) < 1e-7


@pytest.mark.parametrize("nc,dims", [(3, [4, 4, 4, 4]), (2, [6, 4, 3, 5])])
def test_lean_fused_with_projection_vs_oracle(nc, dims):
    """FP32-only storage with the per-update projection on (ASKJA_FP32_LEAN):
    the fused kernel within FP32 tolerance of the oracle."""
    O, u, pi, beta = setup(nc, dims, 17 * nc)
    eps, level, n = 0.02, 6, 4
    want_u, want_p = oracle_leapfrog(O, u, pi, n, eps, level)
    with ab.Engine(nc, dims, beta=beta, dt=eps, level=level, precision="fp32-lean", reunitarise=True) as e:
        e.set_links(u)
        e.set_momenta(pi, 0)
        e.leapfrog(n, eps)
        got = e.get_links()
        assert rel(got, want_u) < 2e-5
        assert rel(e.get_momenta(0), want_p) < 1e-4
        m = got.reshape(-1, nc, nc)
        assert np.abs(np.einsum("lij,lkj->lik", m, m.conj()) - np.eye(nc)).max() < 2e-6
