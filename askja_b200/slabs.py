"""One HMC chain decomposed into x0 slabs over several ranks (one GPU each).

The reference's site order has x0 slowest (structs.h:130-165), so the sites
with one x0 value form a contiguous slab of V3 = V / N0 sites.  Rank r of R
owns the N0/R slabs x0 = r N0/R ... (r+1) N0/R - 1 and holds them in a local
lattice of N0/R + 2 slabs: local slab 0 is a copy of the slab below its range
(owned by rank r-1, periodic), local slab N0/R + 1 a copy of the slab above
(rank r+1).  Every staple of an owned link lies within one slab of it in x0,
so the force on owned links is exact as long as the halo slabs hold the
neighbours' current links.  The halos are therefore exchanged after every
link update (the one step of the leapfrog that changes links); the force and
link-update launches run over the whole local lattice, and what they compute
on the halo slabs is overwritten by the next exchange.

The trajectory uses the reference's own step order (sun.cpp:1174-1318 through
the seam functions updateE / updateUandcopyDown): updateE(dt/2), then per MD
step updateUandcopyDown(dt), halo exchange, updateE(dt or dt/2 at the end).
The Hamiltonian sums are restricted to the owned sites
(askja_set_reduction_range) and summed over ranks in FP64 (all-reduce); the
Metropolis uniform comes from a generator seeded identically on every rank, so
all ranks take the same decision and keep or restore the same configuration.
Momenta are refreshed by each rank for its local lattice (Philox keyed by the
seed, the rank and the trajectory); the halo momenta are never used.

Communication is torch.distributed point-to-point (NCCL between GPUs, gloo on
CPU): the two boundary slabs are sent, the two halos received, as one batch
of send/recv.  `local_engine` is the per-rank engine (askja_b200.Engine on a
GPU); any object with the same methods works, which is how the decomposition
is tested on CPU against a single-domain run.
"""
from __future__ import annotations

import math

import numpy as np


class SlabChain:
    def __init__(self, nc, dims, beta, dt, level, rank, world, local_engine, seed=120351616, group=None,
                 device_buffers=None):
        dims = [int(d) for d in dims]
        if len(dims) < 2 or dims[0] % world or dims[0] // world < 1:
            raise ValueError(f"N0 = {dims[0]} must be a positive multiple of the {world} ranks and DIM >= 2")
        self.nc, self.dims, self.beta, self.dt, self.level = int(nc), dims, float(beta), float(dt), int(level)
        self.rank, self.world, self.group = int(rank), int(world), group
        self.n0_loc = dims[0] // world
        self.v3 = int(np.prod(dims[1:]))
        self.local_dims = [self.n0_loc + 2] + dims[1:]
        self.e = local_engine
        self.seed = int(seed)
        self.ntraj = 0
        self.uniforms = np.random.default_rng(self.seed)  # the same stream on every rank
        self.device_buffers = device_buffers
        # the owned slabs are local slabs 1 .. n0_loc
        self.e.set_reduction_range(self.v3, (self.n0_loc + 1) * self.v3)

    # ---- layout -------------------------------------------------------------
    def owned(self, u_global: np.ndarray) -> np.ndarray:
        """This rank's local lattice (owned slabs plus both halos) cut from a
        global configuration in U-conf layout (V, D, NC, NC)."""
        n0 = self.dims[0]
        x0 = [(self.rank * self.n0_loc - 1 + k) % n0 for k in range(self.n0_loc + 2)]
        u = u_global.reshape(n0, self.v3, *u_global.shape[1:])
        return np.ascontiguousarray(u[x0].reshape(-1, *u_global.shape[1:]))

    def gather_owned(self, local: np.ndarray) -> np.ndarray:
        """The owned slabs of a local-lattice field."""
        return local.reshape(self.n0_loc + 2, self.v3, *local.shape[1:])[1:-1].reshape(-1, *local.shape[1:])

    # ---- communication ------------------------------------------------------
    def _allreduce(self, x: float) -> float:
        if self.world == 1:
            return x
        import torch
        import torch.distributed as dist
        dev = "cuda" if dist.get_backend(self.group) == "nccl" else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, group=self.group)
        return float(t.item())

    def exchange(self):
        """Halo slabs from the neighbouring ranks: local slab 0 <- the last
        owned slab of rank r-1, local slab n0_loc+1 <- the first owned slab of
        rank r+1 (periodic in x0)."""
        v3, n = self.v3, self.n0_loc
        first = self.e.get_slab(1 * v3, v3)
        last = self.e.get_slab(n * v3, v3)
        if self.world == 1:
            self.e.set_slab(0, last)
            self.e.set_slab((n + 1) * v3, first)
            return
        import torch
        import torch.distributed as dist
        nccl = dist.get_backend(self.group) == "nccl"
        dev = "cuda" if nccl else "cpu"
        up, down = (self.rank + 1) % self.world, (self.rank - 1) % self.world
        s_first = torch.from_numpy(first.view(np.float64).ravel()).to(dev)
        s_last = torch.from_numpy(last.view(np.float64).ravel()).to(dev)
        r_below = torch.empty_like(s_first)
        r_above = torch.empty_like(s_first)
        ops = [dist.P2POp(dist.isend, s_last, up, self.group), dist.P2POp(dist.irecv, r_below, down, self.group),
               dist.P2POp(dist.isend, s_first, down, self.group), dist.P2POp(dist.irecv, r_above, up, self.group)]
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        shape = first.shape
        self.e.set_slab(0, r_below.cpu().numpy().view(np.complex128).reshape(shape))
        self.e.set_slab((n + 1) * v3, r_above.cpu().numpy().view(np.complex128).reshape(shape))

    # ---- HMC ---------------------------------------------------------------
    def hamiltonian(self, which: int) -> float:
        """beta (S + K / (2 NC)) of the whole lattice: owned sums, all-reduced."""
        s = self.e.EnergyMag()
        k = self.e.simpleenergyEl(which)
        tot = self._allreduce(s + k / (2.0 * self.nc))
        return self.beta * tot

    def leapfrog(self, nsteps: int, eps: float):
        """updateE(eps/2), then nsteps x (updateUandcopyDown(eps), halo
        exchange, updateE(eps, eps/2 at the end)); Pi holds the final momenta."""
        self.e.updateE(0.5 * eps)
        for i in range(nsteps):
            self.e.updateUandcopyDown(eps)
            self.exchange()
            self.e.updateE(eps if i < nsteps - 1 else 0.5 * eps)

    def trajectory(self, nsteps: int, project: bool = False) -> dict:
        """One HMC trajectory of the whole lattice (sun.cpp:1174-1318)."""
        if project:  # FP32: projected links at the start of every trajectory
            self.e.reunitarise()
            self.exchange()
            self.e.takeconfiguration()
        self.e.initializeE(self.seed + 7919 * self.rank, self.ntraj)
        h_old = self.hamiltonian(0)
        self.leapfrog(nsteps, self.dt)
        h_new = self.hamiltonian(1)
        u = float(self.uniforms.random())
        dh = h_new - h_old
        accepted = h_new < h_old or u < math.exp(min(0.0, -dh))
        if accepted:
            self.e.takeconfiguration()
        else:
            self.e.loadconfiguration()
        self.ntraj += 1
        return {"h_old": h_old, "h_new": h_new, "dh": dh, "u": u, "accepted": bool(accepted)}
