"""The short seam names (askja_force_step, askja_link_step, askja_action,
askja_kinetic, askja_refresh_momenta) and askja_measure, called through the C
ABI, give exactly what the reference-named calls give."""
import ctypes

import numpy as np
import pytest

import askja_b200 as ab
from oracle import Oracle, fields

pytestmark = pytest.mark.gpu


def dbl():
    return ctypes.c_double()


@pytest.mark.parametrize("nc,dims,precision", [(3, [4, 3, 2, 2], "fp64"), (3, [4, 4, 4, 2], "fp32"),
                                               (8, [3, 2, 2], "fp64")])
def test_aliases_match(nc, dims, precision):
    rng = np.random.default_rng(nc + len(dims))
    O = Oracle(nc, dims)
    u = fields.haar(nc, O.vol * O.dim, rng).reshape(O.shape)
    with ab.Engine(nc, dims, beta=2.0 * nc, precision=precision) as a, \
            ab.Engine(nc, dims, beta=2.0 * nc, precision=precision) as b:
        L = a.lib
        for e in (a, b):
            e.set_links(u)
        assert L.askja_refresh_momenta(a._ctx, 5, 7) == 0
        b.initializeE(5, 7)
        assert np.array_equal(a.get_momenta(0), b.get_momenta(0))
        assert L.askja_force_step(a._ctx, ctypes.c_double(0.02)) == 0
        b.updateE(0.02)
        assert np.array_equal(a.get_momenta(1), b.get_momenta(1))
        assert L.askja_link_step(a._ctx, ctypes.c_double(0.02)) == 0
        b.updateUandcopyDown(0.02)
        assert np.array_equal(a.get_links(), b.get_links())
        s, k = dbl(), dbl()
        assert L.askja_action(a._ctx, ctypes.byref(s)) == 0
        assert L.askja_kinetic(a._ctx, ctypes.byref(k)) == 0
        assert s.value == b.EnergyMag()
        assert k.value == b.simpleenergyEl(0)
        m = a.measure()
        t, sp = b.PlaqExp()
        want = [t, sp, b.PolyakovLoop()] + [b.WilsonLoopDir(d) for d in range(1, len(dims))] + [b.GaussLaw(), b.UViol()]
        assert m.tolist() == want


def test_measure_needs_two_dims():
    with ab.Engine(3, [4], beta=1.0) as e:
        out = (ctypes.c_double * 8)()
        assert e.lib.askja_measure(e._ctx, out) == -1  # ASKJA_ERR_ARG
