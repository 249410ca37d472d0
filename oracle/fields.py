"""Test infrastructure only: seeded synthetic gauge and momentum fields in
U-conf layout, shape (V, D, NC, NC) complex128.

* ``haar(nc, nlinks, rng)`` -- Haar-random SU(NC): QR of a complex Gaussian
  matrix with the R-diagonal phase fix (Mezzadri 2007), then the last row
  multiplied by conj(det) so that det = 1.
* ``near_identity(...)`` -- exp(i eps H) for random Hermitian H: a
  "thermalised-like" configuration with plaquettes away from both 0 and 1.
* ``momenta(nc, nlinks, beta, rng, oracle)`` -- the reference's momentum
  distribution P = sqrt(2 NC / beta) sum_a xi_a T_a (sun.cpp:230-247).
"""
from __future__ import annotations

import numpy as np


def haar(nc: int, nlinks: int, rng: np.random.Generator) -> np.ndarray:
    z = (rng.standard_normal((nlinks, nc, nc)) + 1j * rng.standard_normal((nlinks, nc, nc))) / np.sqrt(2.0)
    q, r = np.linalg.qr(z)
    d = np.diagonal(r, axis1=1, axis2=2)
    q = q * (d / np.abs(d))[:, None, :]
    det = np.linalg.det(q)
    q[:, -1, :] *= (np.conj(det) / np.abs(det))[:, None]
    return q


def random_hermitian_traceless(nc: int, nlinks: int, rng: np.random.Generator) -> np.ndarray:
    a = rng.standard_normal((nlinks, nc, nc)) + 1j * rng.standard_normal((nlinks, nc, nc))
    h = 0.5 * (a + np.conj(np.swapaxes(a, 1, 2)))
    tr = np.trace(h, axis1=1, axis2=2) / nc
    h -= tr[:, None, None] * np.eye(nc)[None]
    return h


def near_identity(nc: int, nlinks: int, eps: float, rng: np.random.Generator) -> np.ndarray:
    h = random_hermitian_traceless(nc, nlinks, rng)
    w, v = np.linalg.eigh(h)
    return np.einsum("lij,lj,lkj->lik", v, np.exp(1j * eps * w), np.conj(v))


def momenta(nc: int, nlinks: int, beta: float, rng: np.random.Generator, oracle) -> np.ndarray:
    xi = rng.standard_normal(nlinks * (nc * nc - 1))
    return oracle.momenta_from_normals(xi, beta)
