"""FP32 row-per-thread kernels (5 <= NC <= 64): the Paterson-Stockmeyer drift
(NC <= 8, LEVEL >= 5; Horner below) and the Newton-Schulz projection per
update, against the FP64 oracle, and the gated full reunitarisation that keeps
det U = 1 over many trajectories.

Tolerances are the FP32 path's: relative 5e-5 on the kicked momenta, 1e-5 on
the links after a few fused steps, 2e-6 on the unitarity defect."""
import numpy as np
import pytest

import askja_b200 as ab
from conftest import rel
from oracle import Oracle, fields

pytestmark = pytest.mark.gpu

CASES = [(5, [3, 4, 2], 8), (8, [2, 3, 2, 2], 8), (8, [3, 4, 2], 6), (6, [4, 3], 3), (12, [2, 2, 3], 8)]
IDS = [f"su{n}_{'x'.join(map(str, d))}_L{lv}" for n, d, lv in CASES]


def unitarity(u):
    nc = u.shape[-1]
    m = u.reshape(-1, nc, nc)
    return float(np.max(np.abs(np.conj(np.swapaxes(m, -1, -2)) @ m - np.eye(nc))))


@pytest.mark.parametrize("nc,dims,level", CASES, ids=IDS)
@pytest.mark.parametrize("reunit", [False, True])
def test_leapfrog_vs_oracle(nc, dims, level, reunit):
    rng = np.random.default_rng(nc * 31 + level)
    O = Oracle(nc, dims)
    nl = O.vol * O.dim
    u = fields.haar(nc, nl, rng).reshape(O.shape)
    beta = 2.0 * nc
    pi = fields.momenta(nc, nl, beta, rng, O)
    eps = 0.02
    with ab.Engine(nc, dims, beta=beta, dt=eps, level=level, precision="fp32", reunitarise=reunit,
                   kernel_path=1) as e:
        e.set_links(u)
        e.set_momenta(pi, 0)
        e.leapfrog(4, eps)
        uu, pp = u, O.updateE(u, pi, eps / 2)
        for k in range(4):
            uu = O.updateU(uu, pp, eps, level)
            pp = O.updateE(uu, pp, eps if k < 3 else eps / 2)
        got = e.get_links()
        assert rel(got, uu) < 1e-5
        assert rel(e.get_momenta(0), pp) < 5e-5
        if reunit:
            assert unitarity(got) < 2e-6


def test_trajectories_stay_su_n():
    """200 graph-replayed FP32 SU(8) trajectories: the per-update Newton-Schulz
    step keeps U unitary and the full pass before every 10th trajectory keeps
    det U at 1."""
    nc, dims = 8, [4, 4, 2, 2]
    with ab.Engine(nc, dims, beta=2.0 * nc, dt=0.02, level=8, precision="fp32", seed=9) as e:
        e.hot_start(10)
        last, log = e.run_trajectories(200, 10, use_graph=True)
        assert last["n_tot"] == 200
        assert np.all(np.isfinite(log))
        u = e.get_links().reshape(-1, nc, nc)
        assert unitarity(u) < 2e-6
        assert np.abs(np.linalg.det(u) - 1.0).max() < 5e-6
