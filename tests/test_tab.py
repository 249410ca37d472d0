"""Tab (sun.cpp:580-670) and FourierTrafo (sun.cpp:365-411), diagnostics the
reference defines but never calls.

CPU: the numpy restatement (tab_restated.py, the form the GPU kernels compute)
against the reference's own routines built from its sources (oracle/_ref).
GPU: askja_Tab / askja_Tab_all / askja_FourierTrafo against both.  FP64
throughout; sums taken in a different order agree to 1e-11 relative."""
import numpy as np
import pytest

import askja_b200 as ab
from oracle import Oracle, Reference, fields
from tab_restated import fourier, tab_site

CASES = [(3, [4, 3, 2, 2]), (2, [3, 4, 2]), (4, [2, 3, 2, 3]), (3, [5, 4]), (5, [2, 3, 2])]
IDS = [f"su{n}_{'x'.join(map(str, d))}" for n, d in CASES]

needs_ref = pytest.mark.skipif(not Reference.available(), reason="shim-built reference not available")


def setup(nc, dims, seed):
    rng = np.random.default_rng(seed)
    O = Oracle(nc, dims)
    nl = O.vol * O.dim
    u = fields.haar(nc, nl, rng).reshape(O.shape)
    pi = fields.momenta(nc, nl, 2.0 * nc, rng, O)
    Pi = fields.momenta(nc, nl, 2.0 * nc, rng, O)
    return O, u, pi, Pi


@needs_ref
@pytest.mark.parametrize("nc,dims", CASES, ids=IDS)
def test_restatement_matches_reference(nc, dims):
    O, u, pi, Pi = setup(nc, dims, nc * 7 + len(dims))
    R = Reference(nc, dims, beta=2.0 * nc)
    R.set("u", u)
    R.set("pi", pi)
    R.set("Pi", Pi)
    npt = O.dim + 2
    for i in range(0, O.vol, max(1, O.vol // 5)):
        np.testing.assert_allclose(tab_site(u, pi, Pi, O, i, npt), R.Tab(i, npt), rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(fourier(u, O, nc), R.FourierTrafo(), rtol=1e-12, atol=1e-13)


def _traceless_hermitian(p):
    m = p.reshape(-1, p.shape[-1], p.shape[-1])
    h = 0.5 * (m + np.conj(np.swapaxes(m, 1, 2)))
    h -= np.trace(h, axis1=1, axis2=2)[:, None, None] / m.shape[-1] * np.eye(m.shape[-1])
    return h.reshape(p.shape)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32-lean", "fp32"])
@pytest.mark.parametrize("nc,dims", CASES + [(16, [2, 2, 3]), (40, [3, 2])], ids=IDS + ["su16_2x2x3", "su40_3x2"])
def test_gpu_tab_and_fourier(nc, dims, precision):
    O, u, pi, Pi = setup(nc, dims, nc * 11 + len(dims))
    tol = 1e-11
    if precision != "fp64":  # compare on the FP32-rounded fields the engine holds
        u, pi, Pi = (x.astype(np.complex64).astype(np.complex128) for x in (u, pi, Pi))
        if precision == "fp32" and nc <= 4:
            # residual-plane mode: momenta are held as Hermitian traceless
            # coordinates and Tab reads FP32 matrices made from them
            pi, Pi = _traceless_hermitian(pi), _traceless_hermitian(Pi)
            tol = 2e-6
    npt = min(O.dim + 2, 6)
    with ab.Engine(nc, dims, beta=2.0 * nc, precision=precision) as e:
        e.set_links(u)
        e.set_momenta(pi, 0)
        e.set_momenta(Pi, 1)
        allv = e.Tab_all(npt)
        one = e.Tab(O.vol - 1, npt, mdata=np.ones(npt))
        coef = e.FourierTrafo()
    for i in range(O.vol):
        np.testing.assert_allclose(allv[i], tab_site(u, pi, Pi, O, i, npt), rtol=tol, atol=tol)
    np.testing.assert_allclose(one, 1.0 + allv[O.vol - 1], rtol=1e-14)
    np.testing.assert_allclose(coef, fourier(u, O, nc), rtol=1e-11, atol=1e-12)
    if Reference.available() and nc <= 5 and tol < 1e-10:
        R = Reference(nc, dims, beta=2.0 * nc)
        R.set("u", u)
        R.set("pi", pi)
        R.set("Pi", Pi)
        np.testing.assert_allclose(allv.sum(0), sum(R.Tab(i, npt) for i in range(O.vol)), rtol=1e-11, atol=1e-10)
        np.testing.assert_allclose(coef, R.FourierTrafo(), rtol=1e-11, atol=1e-12)


@pytest.mark.gpu
def test_gpu_tab_arguments():
    with ab.Engine(3, [3, 2, 2], beta=6.0) as e:
        for npt in (1, 6):
            with pytest.raises(ab.AskjaError):
                e.Tab(0, npt)
        with pytest.raises(ab.AskjaError):
            e.Tab(12, 3)
        e.initializeU()
        e.initializeE(1, 0)
        v = e.Tab_all(5)
        # cold start: F = 0, so only the momentum terms remain
        assert np.allclose(v[:, 1], 0.0)
        np.testing.assert_allclose(e.FourierTrafo(), 0.0, atol=1e-14)
