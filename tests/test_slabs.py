"""x0-slab domain decomposition (askja_b200/slabs.py) on CPU: two gloo ranks
(127.0.0.1), each holding its slabs plus halos in a local engine stood in by
the FP64 oracle (test infrastructure), exchange halos after every link update
and all-reduce the Hamiltonian.  The owned links after a leapfrog and the
energies must equal a single-domain oracle leapfrog of the whole lattice to
rounding.  The GPU engine implements the same local-engine methods
(askja_slab, askja_set_reduction_range, the seam calls)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from oracle import Oracle, fields


class OracleLocal:
    """The local-engine methods SlabChain calls, on the FP64 oracle: the local
    lattice is periodic in x0, which only matters on the halo slabs."""

    def __init__(self, nc, dims, beta, level):
        self.O = Oracle(nc, dims)
        self.nc, self.dims, self.beta, self.level = nc, dims, beta, level
        self.r0, self.r1 = 0, self.O.vol
        V, D = self.O.vol, self.O.dim
        self.plus = np.array([[self.O.getplus(s, d) for d in range(D)] for s in range(V)])

    def set_fields(self, u, pi):
        self.u, self.pi, self.Pi, self.uconf = u.copy(), pi.copy(), pi.copy(), u.copy()

    def set_reduction_range(self, s0, s1):
        self.r0, self.r1 = s0, s1

    def get_slab(self, s0, n):
        return self.u[s0:s0 + n].copy()

    def set_slab(self, s0, links):
        self.u[s0:s0 + len(links)] = links

    def updateE(self, eps):
        self.Pi = self.O.updateE(self.u, self.pi, eps)

    def updateUandcopyDown(self, eps):
        self.u = self.O.updateU(self.u, self.Pi, eps, self.level)
        self.pi = self.Pi.copy()

    def EnergyMag(self):
        u, D, tot = self.u, self.O.dim, 0.0
        for s in range(self.r0, self.r1):
            for mu in range(D):
                for nu in range(mu + 1, D):
                    a, b = u[s, mu], u[self.plus[s, mu], nu]
                    c, d = u[self.plus[s, nu], mu], u[s, nu]
                    tot += 1.0 - np.trace(a @ b @ c.conj().T @ d.conj().T).real / self.nc
        return tot

    def simpleenergyEl(self, which):
        p = (self.Pi if which else self.pi)[self.r0:self.r1]
        return float(np.einsum("sdij,sdji->", p, p).real)

    def takeconfiguration(self):
        self.uconf = self.u.copy()

    def loadconfiguration(self):
        self.u = self.uconf.copy()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


NC, DIMS, BETA, EPS, LEVEL, NSTEPS = 3, [4, 3, 2, 2], 5.7, 0.02, 6, 3


def _global_fields():
    rng = np.random.default_rng(41)
    O = Oracle(NC, DIMS)
    u = fields.haar(NC, O.vol * O.dim, rng).reshape(O.shape)
    pi = fields.momenta(NC, O.vol * O.dim, BETA, rng, O)
    return u, pi


def _run_rank(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist

    from askja_b200.slabs import SlabChain

    if world > 1:
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        u, pi = _global_fields()
        n0_loc = DIMS[0] // world
        local = OracleLocal(NC, [n0_loc + 2] + DIMS[1:], BETA, LEVEL)
        chain = SlabChain(NC, DIMS, BETA, EPS, LEVEL, rank, world, local)
        local.set_fields(chain.owned(u), chain.owned(pi))
        h0 = chain.hamiltonian(0)
        chain.leapfrog(NSTEPS, EPS)
        h1 = chain.hamiltonian(1)
        mine = chain.gather_owned(local.u)
        if world > 1:
            parts = [torch.empty(mine.size * 2, dtype=torch.float64) for _ in range(world)]
            dist.all_gather(parts, torch.from_numpy(mine.view(np.float64).ravel().copy()))
            whole = np.concatenate([p.numpy().view(np.complex128) for p in parts]).reshape(u.shape)
        else:
            whole = mine
        q.put((rank, h0, h1, whole))
    finally:
        if world > 1:
            dist.destroy_process_group()


def _expected():
    u, pi = _global_fields()
    O = Oracle(NC, DIMS)
    h0 = BETA * (O.EnergyMag(u) + O.simpleenergyEl(pi) / (2 * NC))
    p = O.updateE(u, pi, 0.5 * EPS)
    for i in range(NSTEPS):
        u = O.updateU(u, p, EPS, LEVEL)
        p = O.updateE(u, p, EPS if i < NSTEPS - 1 else 0.5 * EPS)
    h1 = BETA * (O.EnergyMag(u) + O.simpleenergyEl(p) / (2 * NC))
    return u, h0, h1


@pytest.mark.parametrize("world", [1, 2])
def test_slab_leapfrog_matches_single_domain(world):
    want_u, want_h0, want_h1 = _expected()
    if world == 1:
        import queue
        q = queue.Queue()
        _run_rank(0, 1, 0, q)
        res = [q.get()]
    else:
        ctx = mp.get_context("spawn")
        q = ctx.Queue()
        port = _free_port()
        procs = [ctx.Process(target=_run_rank, args=(r, world, port, q)) for r in range(world)]
        for p in procs:
            p.start()
        res = [q.get(timeout=300) for _ in range(world)]
        for p in procs:
            p.join(timeout=60)
        assert all(p.exitcode == 0 for p in procs)
    for rank, h0, h1, whole in res:
        assert h0 == pytest.approx(want_h0, rel=1e-12)
        assert h1 == pytest.approx(want_h1, rel=1e-12)
        assert np.abs(whole - want_u).max() < 1e-12


def test_slab_layout():
    from askja_b200.slabs import SlabChain
    u, _ = _global_fields()
    v3 = int(np.prod(DIMS[1:]))
    for rank in range(2):
        local = OracleLocal(NC, [4] + DIMS[1:], BETA, LEVEL)
        chain = SlabChain(NC, DIMS, BETA, EPS, LEVEL, rank, 2, local)
        assert (local.r0, local.r1) == (v3, 3 * v3)
        mine = chain.owned(u)
        x0 = [(rank * 2 - 1 + k) % 4 for k in range(4)]
        np.testing.assert_array_equal(mine.reshape(4, v3, *u.shape[1:]), u.reshape(4, v3, *u.shape[1:])[x0])
        np.testing.assert_array_equal(chain.gather_owned(mine), u.reshape(4, v3, *u.shape[1:])[2 * rank:2 * rank + 2]
                                      .reshape(-1, *u.shape[1:]))
    with pytest.raises(ValueError):
        SlabChain(NC, [3, 2, 2], BETA, EPS, LEVEL, 0, 2, OracleLocal(NC, [3, 2, 2], BETA, LEVEL))
