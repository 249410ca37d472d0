"""The autotuner: every candidate mapping computes the same physics (each
is checked against the oracle here), the tuner picks the fastest, leaves u
and pi untouched, and later engines of the same (NC, DIM, precision) start
from the cached choice."""
import numpy as np
import pytest

import askja_b200 as ab
from conftest import rel
from oracle import Oracle, fields

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nc,dims", [(3, [6, 4, 4, 6]), (8, [3, 3, 2, 4])])
def test_every_candidate_matches_oracle(nc, dims):
    rng = np.random.default_rng(nc)
    O = Oracle(nc, dims)
    nl = O.vol * O.dim
    u = fields.haar(nc, nl, rng).reshape(O.shape)
    pi = fields.momenta(nc, nl, 6.0, rng, O)
    with ab.Engine(nc, dims, beta=6.0, dt=0.02, level=6, precision="fp64") as e:
        e.set_links(u)
        e.set_momenta(pi, 0)
        t = ab.autotune(e, reps=2)
        assert t["candidates"] and t["best_us"] == min(c["us"] for c in t["candidates"])
        np.testing.assert_array_equal(e.get_links(), u)
        np.testing.assert_array_equal(e.get_momenta(0), pi)
        want_pi = O.updateE(u, pi, 0.01)
        want_u = O.updateU(u, want_pi, 0.02, 6)
        for cand in t["candidates"]:
            ab.set_tuning(e, cand)
            e.set_links(u)
            e.set_momenta(pi, 0)
            e.leapfrog(1, 0.02)  # kick(eps/2) + drift(eps) + kick(eps/2)
            assert rel(e.get_links(), want_u) < 1e-12, cand
    with ab.Engine(nc, dims, beta=6.0, precision="fp64") as e2:
        # cached: a second autotune-free engine gives identical results to the tuned one
        e2.set_links(u)
        e2.set_momenta(pi, 0)
        e2.updateE(0.01)
        assert rel(e2.get_momenta(1), want_pi) < 1e-12


def test_set_tuning_rejects_nonsense():
    with ab.Engine(8, [2, 2, 2], beta=1.0) as e:
        with pytest.raises(ab.AskjaError):
            ab.set_tuning(e, {"path": 0})  # thread-per-link does not exist for NC = 8


@pytest.mark.parametrize("nc", [5, 8])
def test_fp32_row_register_budgets_agree(nc):
    """The FP32 row kernel for 5 <= NC <= 8 at its three register budgets
    (occupancy 0, 1, 2: 128, 80 and 64 registers, the tighter ones spilling)
    is the same code: identical fields after a few steps, and candidates of the
    autotuner."""
    dims = [3, 2, 4, 4]
    rng = np.random.default_rng(40 + nc)
    O = Oracle(nc, dims)
    nl = O.vol * O.dim
    u = fields.haar(nc, nl, rng).reshape(O.shape)
    pi = fields.momenta(nc, nl, 2.0 * nc, rng, O)
    out = []
    with ab.Engine(nc, dims, beta=2.0 * nc, dt=0.01, level=8, precision="fp32") as e:
        t = ab.autotune(e, reps=2)
        assert {c["occupancy"] for c in t["candidates"] if c["path"] == 1} == {0, 1, 2}
        for occ in (0, 1, 2):
            ab.set_tuning(e, {"path": 1, "occupancy": occ})
            e.set_links(u)
            e.set_momenta(pi, 0)
            e.leapfrog(3, 0.01)
            out.append((e.get_links(), e.get_momenta(0)))
    for links, mom in out[1:]:
        np.testing.assert_array_equal(links, out[0][0])
        np.testing.assert_array_equal(mom, out[0][1])
