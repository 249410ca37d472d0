"""The engine side of the x0-slab decomposition on one GPU: askja_slab and
askja_set_reduction_range, and SlabChain (askja_b200/slabs.py) with one rank,
whose halos are its own boundary slabs (periodic): the owned links and the
energies after a leapfrog equal those of the plain engine on the whole
lattice; and two ranks as two processes on the GPU, exchanging through gloo on
the host.  The exchange logic alone is also tested on CPU (tests/test_slabs.py)."""
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


def _free_port():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


SLAB = dict(nc=3, dims=[4, 4, 4, 4], beta=5.7, eps=0.02, level=6, n=5)


def _gpu_rank(rank, world, port, q, precision):
    """One rank of the slab chain with its own engine on the GPU; the halo
    exchange and the FP64 all-reduce go through gloo on the host."""
    import datetime
    import os

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        c = SLAB
        u, pi = fields_for(c["nc"], c["dims"], 9, c["beta"])
        local_dims = [c["dims"][0] // world + 2] + c["dims"][1:]
        with ab.Engine(c["nc"], local_dims, beta=c["beta"], dt=c["eps"], level=c["level"], precision=precision) as loc:
            chain = SlabChain(c["nc"], c["dims"], c["beta"], c["eps"], c["level"], rank, world, loc)
            loc.set_links(chain.owned(u))
            loc.set_momenta(chain.owned(pi), 0)
            h0 = chain.hamiltonian(0)
            chain.leapfrog(c["n"], c["eps"])
            h1 = chain.hamiltonian(1)
            mine = chain.gather_owned(loc.get_links())
        q.put((rank, h0, h1, mine))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_two_ranks_match_whole_lattice(precision):
    """Two slab ranks as two processes with their own engines (on the one GPU
    a call here has; the ranks' kernels never wait on each other: the halo
    exchange is host-side gloo between MD steps): the owned links and both
    Hamiltonians after a leapfrog equal the whole-lattice engine's."""
    import multiprocessing as mp

    c = SLAB
    u, pi = fields_for(c["nc"], c["dims"], 9, c["beta"])
    with ab.Engine(c["nc"], c["dims"], beta=c["beta"], dt=c["eps"], level=c["level"], precision=precision) as whole:
        whole.set_links(u)
        whole.set_momenta(pi, 0)
        want_h0 = whole.hamiltonian(0)
        whole.updateE(0.5 * c["eps"])
        for i in range(c["n"]):
            whole.updateUandcopyDown(c["eps"])
            whole.updateE(c["eps"] if i < c["n"] - 1 else 0.5 * c["eps"])
        want_h1 = whole.hamiltonian(1)
        want_u = whole.get_links()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gpu_rank, args=(r, 2, port, q, precision)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    got_u = np.concatenate([r[3] for r in res])
    tol = 1e-12 if precision == "fp64" else 1e-6
    assert rel(got_u, want_u) < tol
    for _, h0, h1, _ in res:
        assert h0 == pytest.approx(want_h0, rel=1e-12 if precision == "fp64" else 1e-9)
        assert h1 == pytest.approx(want_h1, rel=1e-12 if precision == "fp64" else 1e-9)
