"""Site-pair mapping (kernel_path 3: FP32 SU(3), the links of two adjacent
sites per thread in packed FP32x2 arithmetic, fields in the site-pair layout
for the length of each MD loop) against the FP64 oracle and against the
thread-per-link FP32 kernel.

Tolerances are those of the FP32 thread-per-link path: relative 5e-5 on the
kicked momenta (the force is a difference of nearly equal staple products)
and 1e-5 on the links; the two FP32 mappings differ only in the order of
their FP32 sums (2e-6 apart after a few steps).  The lattices cover the
neighbour cases of the pair layout: fastest extent 2 (the pair is a whole
row, so both fastest-direction neighbours are the same pair reversed), odd
extents in the other directions, a volume that is not a multiple of the
64-site tile, DIM 2 to 4."""
import numpy as np
import pytest

import askja_b200 as ab
from conftest import rel
from oracle import Oracle, fields

pytestmark = pytest.mark.gpu

CASES = [[4, 4, 4, 6], [3, 5, 4], [5, 2], [3, 3, 2], [2, 3, 2, 8], [6, 4]]
IDS = ["x".join(map(str, d)) for d in CASES]


def setup(dims, seed, beta=5.7):
    rng = np.random.default_rng(seed)
    O = Oracle(3, dims)
    nl = O.vol * O.dim
    u = fields.haar(3, nl, rng).reshape(O.shape)
    pi = fields.momenta(3, nl, beta, rng, O)
    return O, u, pi, beta


def unitarity(u):
    m = u.reshape(-1, 3, 3)
    return float(np.max(np.abs(np.conj(np.swapaxes(m, -1, -2)) @ m - np.eye(3))))


@pytest.mark.parametrize("dims", CASES, ids=IDS)
@pytest.mark.parametrize("reunit", [False, True])
def test_leapfrog_vs_oracle(dims, reunit):
    O, u, pi, beta = setup(dims, 17 + len(dims))
    eps = 0.02
    with ab.Engine(3, dims, beta=beta, dt=eps, level=6, precision="fp32", reunitarise=reunit, kernel_path=3) as e:
        e.set_links(u)
        e.set_momenta(pi, 0)
        e.leapfrog(4, eps)
        uu, pp = u, O.updateE(u, pi, eps / 2)
        for k in range(4):
            uu = O.updateU(uu, pp, eps, 6)
            pp = O.updateE(uu, pp, eps if k < 3 else eps / 2)
        got = e.get_links()
        assert rel(got, uu) < 1e-5
        assert rel(e.get_momenta(0), pp) < 5e-5
        if reunit:
            assert unitarity(got) < 2e-6


@pytest.mark.parametrize("dims", CASES, ids=IDS)
def test_matches_thread_per_link(dims):
    """Same inputs through the thread-per-link FP32 kernel (path 0) and the
    site-pair kernel (path 3): links and momenta after 6 fused steps, and the
    layout is back to canonical after the loop (the getters read it)."""
    O, u, pi, beta = setup(dims, 5 * len(dims) + dims[-1])
    out = {}
    for path in (0, 3):
        with ab.Engine(3, dims, beta=beta, dt=0.02, level=6, precision="fp32", kernel_path=path) as e:
            e.set_links(u)
            e.set_momenta(pi, 0)
            e.leapfrog(6, 0.02)
            out[path] = (e.get_links(), e.get_momenta(0))
    assert rel(out[3][0], out[0][0]) < 2e-6
    assert rel(out[3][1], out[0][1]) < 2e-5


def test_md_steps_matches_thread_per_link():
    """askja_md_steps (drift, fused kick+drift steps, out-of-place last kick):
    pi and Pi agree between the two FP32 mappings."""
    dims = [4, 3, 4, 4]
    O, u, pi, beta = setup(dims, 77)
    Pi = fields.momenta(3, O.vol * O.dim, beta, np.random.default_rng(78), O)
    out = {}
    for path in (0, 3):
        with ab.Engine(3, dims, beta=beta, level=6, precision="fp32", kernel_path=path) as e:
            e.set_links(u)
            e.set_momenta(pi, 0)
            e.set_momenta(Pi, 1)
            e.md_steps(5, 0.02)
            out[path] = (e.get_links(), e.get_momenta(0), e.get_momenta(1))
    for a, b in zip(out[3], out[0]):
        assert rel(a, b) < 2e-5


def test_trajectories_match_thread_per_link():
    """Whole trajectories through the graph replay: the energies and dH of
    the two FP32 mappings agree, and both stay close to the FP64 engine."""
    dims = [4, 4, 4, 6]
    O, u, pi, beta = setup(dims, 3)
    logs = {}
    for path, prec in [(3, "fp32"), (0, "fp32-lean"), (0, "fp64")]:
        with ab.Engine(3, dims, beta=beta, dt=0.02, level=6, precision=prec, kernel_path=path, seed=11) as e:
            e.set_links(u)
            last, log = e.run_trajectories(4, 25, use_graph=True)
            assert last["n_tot"] == 4
            logs[(path, prec)] = log
    a, b, c = logs[(3, "fp32")], logs[(0, "fp32-lean")], logs[(0, "fp64")]
    assert np.all(np.isfinite(a))
    np.testing.assert_allclose(a[:, 0], b[:, 0], rtol=1e-5)
    assert np.abs(a[:, 2] - b[:, 2]).max() < 2e-3
    assert np.abs(a[:, 2] - c[:, 2]).max() < 1e-2


def test_path_validation():
    with pytest.raises(ab.AskjaError):
        ab.Engine(3, [4, 4, 3], beta=1.0, precision="fp32", kernel_path=3)  # odd fastest extent
    with pytest.raises(ab.AskjaError):
        ab.Engine(3, [4, 4], beta=1.0, precision="fp64", kernel_path=3)
    with pytest.raises(ab.AskjaError):
        ab.Engine(2, [4, 4], beta=1.0, precision="fp32", kernel_path=3)
    with pytest.raises(ab.AskjaError):
        ab.Engine(3, [4], beta=1.0, precision="fp32", kernel_path=3)
    with ab.Engine(3, [4, 3], beta=1.0, precision="fp32-lean") as e:
        with pytest.raises(ab.AskjaError):
            ab.set_tuning(e, {"path": 3})
    with ab.Engine(3, [3, 4], beta=1.0, precision="fp32-lean") as e:
        ab.set_tuning(e, {"path": 3})
        ab.set_tuning(e, {"path": 0})
    with ab.Engine(3, [3, 4], beta=1.0, precision="fp32") as e:
        with pytest.raises(ab.AskjaError):  # the residual-plane mode has the thread-per-link mapping only
            ab.set_tuning(e, {"path": 3})


def test_pair_tuning_applied_explicitly():
    """The site-pair mapping is not an autotuner candidate (slower than the
    thread-per-link kernel at every measured volume) but can be applied with
    askja_set_tuning, including its register-budget variant, and trajectories
    run on it."""
    dims = [4, 4, 4, 4]
    O, u, pi, beta = setup(dims, 8)
    with ab.Engine(3, dims, beta=beta, precision="fp32-lean") as e:
        e.set_links(u)
        t = ab.autotune(e, reps=2)
        assert 3 not in [c["path"] for c in t["candidates"]]
        for occ in (0, 1):
            ab.set_tuning(e, {"path": 3, "occupancy": occ})
            r = e.trajectory(5)
            assert np.isfinite(r["dh"])
