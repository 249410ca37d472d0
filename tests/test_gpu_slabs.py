"""The engine side of the x0-slab decomposition on one GPU: askja_slab and
askja_set_reduction_range, and SlabChain (askja_b200/slabs.py) with one rank,
whose halos are its own boundary slabs (periodic): the owned links and the
energies after a leapfrog equal those of the plain engine on the whole
lattice.  The exchange between ranks is tested on CPU (tests/test_slabs.py)."""
import numpy as np
import pytest

import askja_b200 as ab
from askja_b200.slabs import SlabChain
from conftest import rel
from oracle import Oracle, fields

pytestmark = pytest.mark.gpu


def fields_for(nc, dims, seed, beta):
    rng = np.random.default_rng(seed)
    O = Oracle(nc, dims)
    return fields.haar(nc, O.vol * O.dim, rng).reshape(O.shape), fields.momenta(nc, O.vol * O.dim, beta, rng, O)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_slab_copies_and_reduction_range(precision):
    nc, dims, beta = 3, [4, 4, 2, 4], 5.7
    u, pi = fields_for(nc, dims, 3, beta)
    v3 = 32
    with ab.Engine(nc, dims, beta=beta, precision=precision) as e:
        e.set_links(u)
        e.set_momenta(pi, 0)
        full = e.EnergyMag(), e.simpleenergyEl(0)
        got = e.get_slab(v3, 2 * v3)
        tol = 1e-15 if precision == "fp64" else 1e-10
        assert np.abs(got - u[v3:3 * v3]).max() < tol
        parts = []
        for s0, s1 in ((0, 40), (40, 128)):
            e.set_reduction_range(s0, s1)
            parts.append((e.EnergyMag(), e.simpleenergyEl(0)))
        assert sum(p[0] for p in parts) == pytest.approx(full[0], rel=1e-13)
        assert sum(p[1] for p in parts) == pytest.approx(full[1], rel=1e-13)
        e.set_reduction_range(0, 128)
        e.set_slab(0, u[2 * v3:3 * v3])  # slab 2 written over slab 0
        assert np.abs(e.get_links()[:v3] - u[2 * v3:3 * v3]).max() < tol
        with pytest.raises(ab.AskjaError):
            e.set_reduction_range(10, 5)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_single_rank_slab_chain_matches_whole_lattice(precision):
    nc, dims, beta, eps, level, n = 3, [4, 4, 4, 4], 5.7, 0.02, 6, 5
    u, pi = fields_for(nc, dims, 9, beta)
    local_dims = [dims[0] + 2] + dims[1:]
    with ab.Engine(nc, dims, beta=beta, dt=eps, level=level, precision=precision) as whole, \
            ab.Engine(nc, local_dims, beta=beta, dt=eps, level=level, precision=precision) as loc:
        chain = SlabChain(nc, dims, beta, eps, level, 0, 1, loc)
        loc.set_links(chain.owned(u))
        loc.set_momenta(chain.owned(pi), 0)
        whole.set_links(u)
        whole.set_momenta(pi, 0)
        assert chain.hamiltonian(0) == pytest.approx(whole.hamiltonian(0), rel=1e-12)
        chain.leapfrog(n, eps)
        whole.updateE(0.5 * eps)
        for i in range(n):
            whole.updateUandcopyDown(eps)
            whole.updateE(eps if i < n - 1 else 0.5 * eps)
        tol = 1e-12 if precision == "fp64" else 1e-6
        assert rel(chain.gather_owned(loc.get_links()), whole.get_links()) < tol
        assert chain.hamiltonian(1) == pytest.approx(whole.hamiltonian(1), rel=1e-12 if precision == "fp64" else 1e-9)
