"""Test infrastructure only: the FP64 CPU oracle for the askja HMC path.

Two checkers live here and nothing in the product imports them:

* ``Oracle`` -- ctypes wrapper of ``askja_oracle.c``, the project's plain-C
  restatement of the reference's routines (each C function cites the
  reference file:line it follows).
* ``Reference`` -- ctypes wrapper of ``_ref/libref_sun.so`` and
  ``_ref/libref_measure4d.so``: the reference's own ``sun.cpp`` and
  ``measurements4d.cpp`` compiled unchanged against the project-written GSL
  shim by ``oracle/Makefile``.  Only available where the reference sources
  were present at build time.

All arrays use the reference's U-conf layout: float64, shape
``(V, D, NC, NC)`` complex128 (or the equivalent interleaved doubles).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_DIR = os.path.join(HERE, "_ref")
ORACLE_SO = os.path.join(BUILD, "libaskja_oracle.so")
# where the reference sources are read from when oracle/_ref is built (absent: not built)
REFERENCE_ROOT = os.environ.get("ASKJA_REFERENCE", "/root/reference")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build_oracle(force: bool = False) -> str:
    """Compile the C restatement (gcc -O2 -fopenmp) into oracle/_build."""
    src = os.path.join(HERE, "askja_oracle.c")
    os.makedirs(BUILD, exist_ok=True)
    if force or not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.check_call(
            ["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-fvisibility=hidden", "-std=gnu11", src, "-lm",
             "-o", ORACLE_SO])
    return ORACLE_SO


def build_reference(force: bool = False) -> bool:
    """Build oracle/_ref from the reference sources if they are present."""
    if not os.path.isdir(REFERENCE_ROOT):
        return False
    args = ["make", "-C", HERE, f"REF={REFERENCE_ROOT}"]
    if force:
        args.append("-B")
    subprocess.check_call(args, stdout=subprocess.DEVNULL)
    return True


def _c(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _dims(n):
    arr = (ctypes.c_int * len(n))(*n)
    return arr


def as_doubles(x: np.ndarray) -> np.ndarray:
    """complex128 array -> contiguous interleaved float64 view."""
    x = np.ascontiguousarray(x, dtype=np.complex128)
    return x.view(np.float64)


class Oracle:
    """FP64 CPU restatement of the reference path (askja_oracle.c)."""

    def __init__(self, nc: int, dims):
        self.lib = ctypes.CDLL(build_oracle())
        self.nc = int(nc)
        self.dims = [int(d) for d in dims]
        self.dim = len(self.dims)
        self.vol = int(np.prod(self.dims))
        L = self.lib
        for name in ("or_EnergyMag", "or_simpleenergyEl", "or_UViol", "or_WilsonLoop_sun", "or_PolyakovLoop"):
            getattr(L, name).restype = ctypes.c_double
        L.or_EnergyEl.restype = ctypes.c_double
        L.or_GaussLaw.restype = ctypes.c_double
        L.or_WilsonLoopDir.restype = ctypes.c_double
        L.or_updateE.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _dp, _dp, ctypes.c_double, _dp]
        L.or_updateU.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _dp, _dp, ctypes.c_double, ctypes.c_int, _dp]
        L.or_getplus.restype = ctypes.c_long
        L.or_getminus.restype = ctypes.c_long
        L.or_getplus.argtypes = [ctypes.c_int, _ip, ctypes.c_long, ctypes.c_int]
        L.or_getminus.argtypes = [ctypes.c_int, _ip, ctypes.c_long, ctypes.c_int]
        L.or_engine_normals.argtypes = [ctypes.c_int, ctypes.c_long, ctypes.c_uint64, ctypes.c_uint64, _dp]
        L.or_momenta_from_normals.argtypes = [ctypes.c_int, ctypes.c_long, ctypes.c_double, _dp, _dp]
        self._n = _dims(self.dims)

    @property
    def shape(self):
        return (self.vol, self.dim, self.nc, self.nc)

    def _in(self, x):
        x = np.ascontiguousarray(x, dtype=np.complex128).reshape(self.shape)
        return x, _c(x.view(np.float64))

    def updateE(self, u, pi, eps):
        u, up = self._in(u)
        pi, pp = self._in(pi)
        out = np.empty(self.shape, np.complex128)
        rc = self.lib.or_updateE(self.nc, self.dim, self._n, up, pp, float(eps), _c(out.view(np.float64)))
        assert rc == 0
        return out

    def updateU(self, u, Pi, eps, level):
        u, up = self._in(u)
        Pi, pp = self._in(Pi)
        out = np.empty(self.shape, np.complex128)
        rc = self.lib.or_updateU(self.nc, self.dim, self._n, up, pp, float(eps), int(level), _c(out.view(np.float64)))
        assert rc == 0
        return out

    def EnergyMag(self, u):
        u, up = self._in(u)
        return self.lib.or_EnergyMag(self.nc, self.dim, self._n, up)

    def simpleenergyEl(self, p):
        p, pp = self._in(p)
        return self.lib.or_simpleenergyEl(self.nc, self.dim, self._n, pp)

    def EnergyEl(self, pi, Pi):
        pi, a = self._in(pi)
        Pi, b = self._in(Pi)
        return self.lib.or_EnergyEl(self.nc, self.dim, self._n, a, b)

    def GaussLaw(self, u, Pi):
        u, a = self._in(u)
        Pi, b = self._in(Pi)
        return self.lib.or_GaussLaw(self.nc, self.dim, self._n, a, b)

    def UViol(self, u):
        u, a = self._in(u)
        return self.lib.or_UViol(self.nc, self.dim, self._n, a)

    def WilsonLoop_sun(self, u):
        u, a = self._in(u)
        return self.lib.or_WilsonLoop_sun(self.nc, self.dim, self._n, a)

    def PolyakovLoop(self, u):
        u, a = self._in(u)
        return self.lib.or_PolyakovLoop(self.nc, self.dim, self._n, a)

    def WilsonLoopDir(self, u, d):
        u, a = self._in(u)
        return self.lib.or_WilsonLoopDir(self.nc, self.dim, self._n, a, int(d))

    def PlaqExp(self, u):
        u, a = self._in(u)
        t, s = ctypes.c_double(), ctypes.c_double()
        rc = self.lib.or_PlaqExp(self.nc, self.dim, self._n, a, ctypes.byref(t), ctypes.byref(s))
        assert rc == 0
        return t.value, s.value

    def scalarLoopcorr(self, u):
        u, a = self._in(u)
        out = np.zeros(self.dims[0])
        self.lib.or_scalarLoopcorr(self.nc, self.dim, self._n, a, _c(out))
        return out

    def getplus(self, ind, d):
        return self.lib.or_getplus(self.dim, self._n, int(ind), int(d))

    def getminus(self, ind, d):
        return self.lib.or_getminus(self.dim, self._n, int(ind), int(d))

    def generators(self):
        out = np.zeros((self.nc * self.nc - 1, self.nc, self.nc), np.complex128)
        self.lib.or_generators(self.nc, _c(out.view(np.float64)))
        return out

    def momenta_from_normals(self, xi, beta):
        xi = np.ascontiguousarray(xi, dtype=np.float64)
        nl = xi.size // (self.nc * self.nc - 1)
        out = np.zeros((nl, self.nc, self.nc), np.complex128)
        self.lib.or_momenta_from_normals(self.nc, nl, float(beta), _c(xi), _c(out.view(np.float64)))
        return out.reshape(self.shape)

    def engine_normals(self, seed, traj):
        nl = self.vol * self.dim
        xi = np.zeros(nl * (self.nc * self.nc - 1))
        self.lib.or_engine_normals(self.nc, nl, int(seed), int(traj), _c(xi))
        return xi

    def mexpi(self, a, level):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        out = np.zeros_like(a)
        self.lib.or_mexpi(self.nc, _c(a.view(np.float64)), int(level), _c(out.view(np.float64)))
        return out

    def adjoint(self, a):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        out = np.zeros_like(a)
        self.lib.or_adjoint(self.nc, _c(a.view(np.float64)), _c(out.view(np.float64)))
        return out

    def reunitarise(self, a):
        a = np.array(a, dtype=np.complex128, copy=True, order="C")
        flat = a.reshape(-1, self.nc, self.nc)
        for m in flat:
            self.lib.or_reunitarise(self.nc, _c(m.view(np.float64)))
        return a


class Reference:
    """The reference's own routines (sun.cpp, measurements4d.cpp) via oracle/_ref."""

    SUN = os.path.join(REF_DIR, "libref_sun.so")
    MEAS = os.path.join(REF_DIR, "libref_measure4d.so")

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(cls.SUN) and os.path.exists(cls.MEAS)

    def __init__(self, nc: int, dims, beta: float = 1.0, level: int = 8):
        if not self.available():
            raise RuntimeError("oracle/_ref not built (needs the reference sources)")
        mode = getattr(os, "RTLD_LOCAL", 0) | getattr(os, "RTLD_NOW", 2)
        self.sun = ctypes.CDLL(self.SUN, mode=mode)
        self.meas = ctypes.CDLL(self.MEAS, mode=mode)
        self.nc = int(nc)
        self.dims = [int(d) for d in dims]
        self.dim = len(self.dims)
        self.vol = int(np.prod(self.dims))
        S, M = self.sun, self.meas
        for f in ("ref_EnergyMag", "ref_simpleenergyEl", "ref_EnergyEl", "ref_TotalEnergy", "ref_GaussLaw",
                  "ref_UViol", "ref_WilsonLoop"):
            getattr(S, f).restype = ctypes.c_double
        S.ref_updateE.argtypes = [ctypes.c_double]
        S.ref_updateUandcopyDown.argtypes = [ctypes.c_double]
        S.ref_init.argtypes = [ctypes.c_int, ctypes.c_int, _ip, ctypes.c_double, ctypes.c_int]
        S.ref_getplus.restype = ctypes.c_long
        S.ref_getminus.restype = ctypes.c_long
        S.ref_getplus.argtypes = [ctypes.c_long, ctypes.c_int]
        S.ref_getminus.argtypes = [ctypes.c_long, ctypes.c_int]
        M.refm_init.argtypes = [ctypes.c_int, ctypes.c_int, _ip, ctypes.c_double]
        M.refm_PolyakovLoop.restype = ctypes.c_double
        M.refm_WilsonLoop.restype = ctypes.c_double
        n = _dims(self.dims)
        assert S.ref_init(self.nc, self.dim, n, float(beta), int(level)) == 0
        assert M.refm_init(self.nc, self.dim, n, float(beta)) == 0

    @property
    def shape(self):
        return (self.vol, self.dim, self.nc, self.nc)

    FIELDS = {"u": 0, "U": 1, "pi": 2, "Pi": 3, "uconf": 4}

    def set(self, name, x):
        x = np.ascontiguousarray(x, dtype=np.complex128).reshape(self.shape)
        assert self.sun.ref_set_field(self.FIELDS[name], _c(x.view(np.float64))) == 0
        if name == "u":
            assert self.meas.refm_set_u(_c(x.view(np.float64))) == 0

    def get(self, name):
        out = np.empty(self.shape, np.complex128)
        assert self.sun.ref_get_field(self.FIELDS[name], _c(out.view(np.float64))) == 0
        return out

    def threads(self, n):
        self.sun.ref_set_threads(int(n))

    def updateE(self, eps):
        self.sun.ref_updateE(float(eps))

    def updateUandcopyDown(self, eps):
        self.sun.ref_updateUandcopyDown(float(eps))

    def EnergyMag(self):
        return self.sun.ref_EnergyMag()

    def simpleenergyEl(self, which="pi"):
        return self.sun.ref_simpleenergyEl(self.FIELDS[which])

    def EnergyEl(self):
        return self.sun.ref_EnergyEl()

    def GaussLaw(self):
        return self.sun.ref_GaussLaw()

    def UViol(self):
        return self.sun.ref_UViol()

    def WilsonLoop_sun(self):
        return self.sun.ref_WilsonLoop()

    def PolyakovLoop(self):
        return self.meas.refm_PolyakovLoop()

    def WilsonLoopDir(self, d):
        return self.meas.refm_WilsonLoop(int(d))

    def PlaqExp(self):
        t, s = ctypes.c_double(), ctypes.c_double()
        self.meas.refm_PlaqExp(ctypes.byref(t), ctypes.byref(s))
        return t.value, s.value

    def scalarLoopcorr(self):
        out = np.zeros(self.dims[0])
        self.meas.refm_scalarLoopcorr(_c(out))
        return out

    def generators(self):
        out = np.zeros((self.nc * self.nc - 1, self.nc, self.nc), np.complex128)
        self.sun.ref_generators(_c(out.view(np.float64)))
        return out

    def mexpi(self, a, level):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        out = np.zeros_like(a)
        self.sun.ref_mexpi(_c(a.view(np.float64)), int(level), _c(out.view(np.float64)))
        return out

    def adjoint(self, a):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        out = np.zeros_like(a)
        self.sun.ref_Adjoint(_c(a.view(np.float64)), _c(out.view(np.float64)))
        return out

    def Tab(self, i, npt, mdata=None):
        m = np.zeros(npt) if mdata is None else np.ascontiguousarray(mdata, dtype=np.float64)
        self.sun.ref_Tab(ctypes.c_long(int(i)), _c(m), ctypes.c_int(int(npt)))
        return m

    def FourierTrafo(self):
        out = np.zeros(self.dims[0])
        self.sun.ref_FourierTrafo(_c(out))
        return out

    def getplus(self, ind, d):
        return self.sun.ref_getplus(int(ind), int(d))

    def getminus(self, ind, d):
        return self.sun.ref_getminus(int(ind), int(d))
