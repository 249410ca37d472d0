"""askja_b200 -- Python mirror of the askja B200 engine's C ABI.

The engine itself is ``libaskja_b200.so`` (CUDA, sm_100a), declared in
``include/askja_gpu.h``.  This module only binds it with ctypes and mirrors
the reference's in-process seam under the reference's own names
(paro8929/askja sun.cpp: ``updateE``, ``updateUandcopyDown``, ``copyDown``,
``EnergyMag``, ``simpleenergyEl``, ``EnergyEl``, ``TotalEnergy``,
``GaussLaw``, ``UViol``, ``WilsonLoop``, ``takeconfiguration``,
``loadconfiguration``, ``initializeU``, ``initializeE``; measurements4d.cpp:
``PolyakovLoop``, ``WilsonLoop(dir)``, ``PlaqExp``, ``scalarLoopcorr``).

Arrays are numpy complex128 in the reference's U-conf order, shape
``(V, DIM, NC, NC)`` with the site index x0-slowest.  There is no CPU
fallback: a missing library or a missing GPU raises ``AskjaError``.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libaskja_b200.so")
EXE_PATH = os.path.join(HERE, "askja")

ASKJA_OK = 0
ERRORS = {-1: "ASKJA_ERR_ARG", -2: "ASKJA_ERR_CUDA", -3: "ASKJA_ERR_IO", -4: "ASKJA_ERR_NONFINITE",
          -5: "ASKJA_ERR_NODEVICE", -6: "ASKJA_ERR_PARSE"}
FP64, FP32, FP32_LEAN = 0, 1, 2
PRECISIONS = {"fp64": FP64, "fp32": FP32, "fp32-lean": FP32_LEAN}
MAX_DIM = 16

# every entry point include/askja_gpu.h declares
EXPORTS = [
    "askja_create", "askja_destroy", "askja_last_error", "askja_version", "askja_volume", "askja_stream",
    "askja_sync", "askja_set_links", "askja_get_links", "askja_get_saved_links", "askja_set_momenta",
    "askja_get_momenta", "askja_initializeU", "askja_hot_start", "askja_initializeE", "askja_updateE",
    "askja_updateUandcopyDown", "askja_copyDown", "askja_takeconfiguration", "askja_loadconfiguration",
    "askja_reunitarise", "askja_EnergyMag", "askja_simpleenergyEl", "askja_EnergyEl", "askja_TotalEnergy",
    "askja_GaussLaw", "askja_UViol", "askja_WilsonLoop", "askja_PolyakovLoop", "askja_WilsonLoopDir",
    "askja_PlaqExp", "askja_scalarLoopcorr", "askja_eigenphases", "askja_trajectory", "askja_run_trajectories", "askja_leapfrog",
    "askja_md_steps", "askja_params_load", "askja_params_store", "askja_file_stem", "askja_conf_write",
    "askja_conf_read", "askja_host_alloc", "askja_host_free", "askja_plaqexp_static", "askja_tc_wait_selftest", "askja_set_reduction_range", "askja_slab",
    "askja_batch_create", "askja_batch_destroy", "askja_batch_last_error", "askja_batch_stream",
    "askja_batch_hot_start", "askja_batch_set_links", "askja_batch_get_links", "askja_batch_run",
    "askja_batch_plaquette", "askja_autotune", "askja_set_tuning", "askja_set_links_async", "askja_trajectory_async",
    "askja_FourierTrafo", "askja_Tab", "askja_Tab_all",
    "askja_force_step", "askja_link_step", "askja_action", "askja_kinetic", "askja_refresh_momenta", "askja_measure",
]


class AskjaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [("nc", ctypes.c_int), ("dim", ctypes.c_int), ("n", ctypes.c_int * MAX_DIM),
                ("beta", ctypes.c_double), ("dt", ctypes.c_double), ("level", ctypes.c_int),
                ("precision", ctypes.c_int), ("reunitarise", ctypes.c_int), ("device", ctypes.c_int),
                ("kernel_path", ctypes.c_int), ("seed", ctypes.c_uint64)]


class TrajResult(ctypes.Structure):
    _fields_ = [("h_old", ctypes.c_double), ("h_new", ctypes.c_double), ("dh", ctypes.c_double),
                ("u", ctypes.c_double), ("accepted", ctypes.c_int), ("pad", ctypes.c_int),
                ("traj", ctypes.c_ulonglong), ("n_acc", ctypes.c_ulonglong), ("n_acc1", ctypes.c_ulonglong),
                ("n_rej", ctypes.c_ulonglong), ("n_tot", ctypes.c_ulonglong)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_ if f != "pad"}


class RunParams(ctypes.Structure):
    _fields_ = [("nc", ctypes.c_int), ("dim", ctypes.c_int), ("n", ctypes.c_int * MAX_DIM),
                ("beta", ctypes.c_double), ("dt", ctypes.c_double)] + [
        (k, ctypes.c_int) for k in ("steps", "update", "update2", "conftake", "level", "verbose", "runcontinue",
                                    "random", "start", "taken", "nacc", "nac1", "nrec", "ntot")]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_ if f != "n"}
        d["n"] = list(self.n)[: self.dim]
        return d


_lib = None


def library() -> ctypes.CDLL:
    """Load libaskja_b200.so (built in-tree by askja_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise AskjaError(-5, f"{LIB_PATH} is not built; run `python -m askja_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    dp, vp, ip = ctypes.POINTER(ctypes.c_double), ctypes.c_void_p, ctypes.c_int
    L.askja_create.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(vp)]
    L.askja_destroy.argtypes = [vp]
    L.askja_destroy.restype = None
    L.askja_last_error.argtypes = [vp]
    L.askja_last_error.restype = ctypes.c_char_p
    L.askja_version.restype = ctypes.c_char_p
    L.askja_volume.argtypes = [vp]
    L.askja_volume.restype = ctypes.c_long
    L.askja_stream.argtypes = [vp]
    L.askja_stream.restype = vp
    for name in ("askja_sync", "askja_initializeU", "askja_copyDown", "askja_takeconfiguration",
                 "askja_loadconfiguration", "askja_reunitarise"):
        getattr(L, name).argtypes = [vp]
    for name in ("askja_set_links", "askja_set_links_async", "askja_get_links", "askja_get_saved_links"):
        getattr(L, name).argtypes = [vp, vp]
    for name in ("askja_set_momenta", "askja_get_momenta"):
        getattr(L, name).argtypes = [vp, ip, vp]
    L.askja_hot_start.argtypes = [vp, ctypes.c_uint64]
    L.askja_initializeE.argtypes = [vp, ctypes.c_uint64, ctypes.c_uint64]
    for name in ("askja_updateE", "askja_updateUandcopyDown"):
        getattr(L, name).argtypes = [vp, ctypes.c_double]
    for name in ("askja_EnergyMag", "askja_EnergyEl", "askja_TotalEnergy", "askja_GaussLaw", "askja_UViol",
                 "askja_WilsonLoop", "askja_PolyakovLoop", "askja_scalarLoopcorr"):
        getattr(L, name).argtypes = [vp, dp]
    L.askja_simpleenergyEl.argtypes = [vp, ip, dp]
    L.askja_WilsonLoopDir.argtypes = [vp, ip, dp]
    L.askja_PlaqExp.argtypes = [vp, dp, dp]
    L.askja_eigenphases.argtypes = [vp, dp, dp]
    L.askja_FourierTrafo.argtypes = [vp, dp]
    for name in ("askja_force_step", "askja_link_step"):
        getattr(L, name).argtypes = [vp, ctypes.c_double]
    for name in ("askja_action", "askja_kinetic", "askja_measure"):
        getattr(L, name).argtypes = [vp, dp]
    L.askja_refresh_momenta.argtypes = [vp, ctypes.c_uint64, ctypes.c_uint64]
    L.askja_Tab.argtypes = [vp, ctypes.c_long, dp, ip]
    L.askja_Tab_all.argtypes = [vp, ip, dp]
    L.askja_trajectory.argtypes = [vp, ip, ctypes.POINTER(TrajResult)]
    L.askja_trajectory_async.argtypes = [vp, ip, vp]
    L.askja_run_trajectories.argtypes = [vp, ip, ip, ip, ctypes.POINTER(TrajResult), dp]
    L.askja_leapfrog.argtypes = [vp, ip, ctypes.c_double]
    L.askja_md_steps.argtypes = [vp, ip, ctypes.c_double]
    L.askja_tc_wait_selftest.argtypes = [vp, ctypes.c_longlong]
    L.askja_set_reduction_range.argtypes = [vp, ctypes.c_long, ctypes.c_long]
    L.askja_slab.argtypes = [vp, ctypes.c_long, ctypes.c_long, vp, ip]
    L.askja_params_load.argtypes = [ctypes.c_char_p, ctypes.POINTER(RunParams)]
    L.askja_params_store.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(RunParams), ip, ip]
    L.askja_file_stem.argtypes = [ctypes.POINTER(RunParams), ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                  ctypes.c_size_t]
    L.askja_conf_write.argtypes = [ctypes.c_char_p, dp, ctypes.c_long]
    L.askja_conf_read.argtypes = [ctypes.c_char_p, dp, ctypes.c_long]
    L.askja_host_alloc.argtypes = [ctypes.c_size_t]
    L.askja_host_alloc.restype = vp
    L.askja_host_free.argtypes = [vp]
    L.askja_host_free.restype = None
    _lib = L
    return L


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Engine:
    """One askja context: device copies of the reference's globals u, pi, Pi,
    uconf for one lattice, plus a CUDA stream."""

    def __init__(self, nc: int, dims, beta: float, dt: float = 0.02, level: int = 8, precision: str = "fp64",
                 reunitarise: bool | None = None, device: int = 0, seed: int = 120351616, kernel_path: int = 0):
        self.lib = library()
        dims = [int(d) for d in dims]
        p = Params()
        p.nc, p.dim = int(nc), len(dims)
        for i, d in enumerate(dims):
            p.n[i] = d
        p.beta, p.dt, p.level = float(beta), float(dt), int(level)
        p.precision = PRECISIONS[precision]
        p.reunitarise = -1 if reunitarise is None else int(bool(reunitarise))
        p.device, p.kernel_path, p.seed = int(device), int(kernel_path), int(seed)
        self.params = p
        self._ctx = ctypes.c_void_p()
        rc = self.lib.askja_create(ctypes.byref(p), ctypes.byref(self._ctx))
        if rc != ASKJA_OK:
            raise AskjaError(rc, self.lib.askja_last_error(None).decode())
        self.nc, self.dims, self.dim = int(nc), dims, len(dims)
        self.vol = int(np.prod(dims))
        self.beta, self.dt, self.level, self.precision = float(beta), float(dt), int(level), precision

    # -- plumbing --------------------------------------------------------
    @property
    def shape(self):
        return (self.vol, self.dim, self.nc, self.nc)

    def _ck(self, rc: int):
        if rc != ASKJA_OK:
            raise AskjaError(rc, self.lib.askja_last_error(self._ctx).decode())

    def close(self):
        if self._ctx:
            self.lib.askja_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream_ptr(self) -> int:
        return int(self.lib.askja_stream(self._ctx) or 0)

    def sync(self):
        self._ck(self.lib.askja_sync(self._ctx))

    def set_reduction_range(self, s0: int, s1: int):
        """askja_set_reduction_range: only sites [s0, s1) enter the sums."""
        self._ck(self.lib.askja_set_reduction_range(self._ctx, int(s0), int(s1)))

    def get_slab(self, s0: int, nsites: int) -> np.ndarray:
        """askja_slab to host: links of sites [s0, s0 + nsites), U-conf layout."""
        out = np.empty((nsites, self.dim, self.nc, self.nc), np.complex128)
        self._ck(self.lib.askja_slab(self._ctx, int(s0), int(nsites), out.ctypes.data, 1))
        return out

    def set_slab(self, s0: int, links) -> None:
        """askja_slab from host: links of sites [s0, s0 + len(links))."""
        a = np.ascontiguousarray(links, dtype=np.complex128).reshape(-1, self.dim, self.nc, self.nc)
        self._ck(self.lib.askja_slab(self._ctx, int(s0), a.shape[0], a.ctypes.data, 0))

    def slab_device(self, s0: int, nsites: int, ptr: int, to_buf: bool) -> None:
        """askja_slab with a device buffer (e.g. a torch CUDA tensor's data_ptr)."""
        self._ck(self.lib.askja_slab(self._ctx, int(s0), int(nsites), int(ptr), 1 if to_buf else 0))

    def tc_wait_selftest(self, cycles: int):
        """askja_tc_wait_selftest: enqueue the tensor-core path's bounded wait
        on an mbarrier nothing completes; the next sync() raises."""
        self._ck(self.lib.askja_tc_wait_selftest(self._ctx, int(cycles)))

    def _host(self, x):
        x = np.ascontiguousarray(x, dtype=np.complex128).reshape(self.shape)
        return x

    # -- fields ------------------------------------------------------------
    def set_links(self, u):
        u = self._host(u)
        self._ck(self.lib.askja_set_links(self._ctx, u.ctypes.data))

    def set_links_ptr(self, ptr: int):
        """Upload links from a raw host pointer (e.g. pinned memory)."""
        self._ck(self.lib.askja_set_links(self._ctx, ctypes.c_void_p(ptr)))

    def set_links_async(self, ptr: int):
        """askja_set_links_async from a raw (page-locked) host pointer: the copy
        overlaps the work already enqueued; see include/askja_gpu.h."""
        self._ck(self.lib.askja_set_links_async(self._ctx, ctypes.c_void_p(ptr)))

    def get_links(self):
        out = np.empty(self.shape, np.complex128)
        self._ck(self.lib.askja_get_links(self._ctx, out.ctypes.data))
        return out

    def get_saved_links(self):
        out = np.empty(self.shape, np.complex128)
        self._ck(self.lib.askja_get_saved_links(self._ctx, out.ctypes.data))
        return out

    def set_momenta(self, p, which: int = 0):
        p = self._host(p)
        self._ck(self.lib.askja_set_momenta(self._ctx, int(which), p.ctypes.data))

    def get_momenta(self, which: int = 0):
        out = np.empty(self.shape, np.complex128)
        self._ck(self.lib.askja_get_momenta(self._ctx, int(which), out.ctypes.data))
        return out

    def initializeU(self):
        self._ck(self.lib.askja_initializeU(self._ctx))

    def hot_start(self, seed: int):
        self._ck(self.lib.askja_hot_start(self._ctx, int(seed)))

    def initializeE(self, seed: int, counter: int = 0):
        self._ck(self.lib.askja_initializeE(self._ctx, int(seed), int(counter)))

    # -- the reference seam -------------------------------------------------
    def updateE(self, eps: float):
        self._ck(self.lib.askja_updateE(self._ctx, float(eps)))

    def updateUandcopyDown(self, eps: float):
        self._ck(self.lib.askja_updateUandcopyDown(self._ctx, float(eps)))

    def copyDown(self):
        self._ck(self.lib.askja_copyDown(self._ctx))

    def takeconfiguration(self):
        self._ck(self.lib.askja_takeconfiguration(self._ctx))

    def loadconfiguration(self):
        self._ck(self.lib.askja_loadconfiguration(self._ctx))

    def reunitarise(self):
        self._ck(self.lib.askja_reunitarise(self._ctx))

    def _scalar(self, fn, *args):
        v = ctypes.c_double()
        self._ck(fn(self._ctx, *args, ctypes.byref(v)))
        return v.value

    def EnergyMag(self):
        return self._scalar(self.lib.askja_EnergyMag)

    def simpleenergyEl(self, which: int = 0):
        return self._scalar(self.lib.askja_simpleenergyEl, int(which))

    def EnergyEl(self):
        return self._scalar(self.lib.askja_EnergyEl)

    def TotalEnergy(self):
        return self._scalar(self.lib.askja_TotalEnergy)

    def GaussLaw(self):
        return self._scalar(self.lib.askja_GaussLaw)

    def UViol(self):
        return self._scalar(self.lib.askja_UViol)

    def WilsonLoop(self):
        """sun.cpp's WilsonLoop: the line along dir 0 from site 0."""
        return self._scalar(self.lib.askja_WilsonLoop)

    def PolyakovLoop(self):
        return self._scalar(self.lib.askja_PolyakovLoop)

    def WilsonLoopDir(self, d: int):
        return self._scalar(self.lib.askja_WilsonLoopDir, int(d))

    def PlaqExp(self):
        t, s = ctypes.c_double(), ctypes.c_double()
        self._ck(self.lib.askja_PlaqExp(self._ctx, ctypes.byref(t), ctypes.byref(s)))
        return t.value, s.value

    def eigenphases(self):
        """getevs (measurements4d.cpp:185-309): averaged sorted eigenphases of
        the Wilson lines (direction 1) and the Polyakov lines (direction 0)."""
        w, p = np.zeros(self.nc), np.zeros(self.nc)
        self._ck(self.lib.askja_eigenphases(self._ctx, _dptr(w), _dptr(p)))
        return w, p

    def scalarLoopcorr(self):
        out = np.zeros(self.dims[0])
        self._ck(self.lib.askja_scalarLoopcorr(self._ctx, _dptr(out)))
        return out

    def measure(self):
        """askja_measure: [plaq_t, plaq_s, polyakov, wilson(1..DIM-1), gauss, uviol]."""
        out = np.zeros(self.dim + 4)
        self._ck(self.lib.askja_measure(self._ctx, _dptr(out)))
        return out

    def FourierTrafo(self):
        """askja_FourierTrafo: |inverse DFT| of the plaquette energy of sites 0..N0-1."""
        out = np.zeros(self.dims[0])
        self._ck(self.lib.askja_FourierTrafo(self._ctx, _dptr(out)))
        return out

    def Tab(self, site: int, npt: int, mdata=None):
        """askja_Tab: add site's energy-momentum tensor terms to mdata (zeros if None)."""
        m = np.zeros(npt) if mdata is None else np.ascontiguousarray(mdata, dtype=np.float64)
        self._ck(self.lib.askja_Tab(self._ctx, int(site), _dptr(m), int(npt)))
        return m

    def Tab_all(self, npt: int):
        """askja_Tab_all: per-site contributions, shape (V, npt)."""
        out = np.zeros((self.vol, npt))
        self._ck(self.lib.askja_Tab_all(self._ctx, int(npt), _dptr(out)))
        return out

    def hamiltonian(self, which: int = 0):
        """beta * (EnergyMag + simpleenergyEl / (2 NC)), sun.cpp:1175/1254."""
        return self.beta * (self.EnergyMag() + self.simpleenergyEl(which) / (2 * self.nc))

    # -- trajectories ---------------------------------------------------------
    def trajectory(self, nsteps: int) -> dict:
        r = TrajResult()
        self._ck(self.lib.askja_trajectory(self._ctx, int(nsteps), ctypes.byref(r)))
        return r.as_dict()

    def trajectory_async(self, nsteps: int, out_ptr: int = 0):
        """askja_trajectory_async: enqueue a trajectory (graph replay) and the
        copy of its outcome to out_ptr (a page-locked TrajResult, or 0);
        valid after sync()."""
        self._ck(self.lib.askja_trajectory_async(self._ctx, int(nsteps), ctypes.c_void_p(out_ptr or None)))

    def run_trajectories(self, ntraj: int, nsteps: int, use_graph: bool = True, want_log: bool = True):
        r = TrajResult()
        log = np.zeros(4 * max(ntraj, 1)) if want_log else None
        self._ck(self.lib.askja_run_trajectories(self._ctx, int(ntraj), int(nsteps), int(bool(use_graph)),
                                                 ctypes.byref(r), _dptr(log) if log is not None else None))
        return r.as_dict(), (log.reshape(-1, 4)[:ntraj] if log is not None else None)

    def leapfrog(self, nsteps: int, eps: float):
        self._ck(self.lib.askja_leapfrog(self._ctx, int(nsteps), float(eps)))

    def md_steps(self, nsteps: int, eps: float):
        self._ck(self.lib.askja_md_steps(self._ctx, int(nsteps), float(eps)))


# -- host I/O (no GPU needed) ---------------------------------------------------
def params_load(path: str) -> dict:
    L = library()
    rp = RunParams()
    rc = L.askja_params_load(path.encode(), ctypes.byref(rp))
    if rc != ASKJA_OK:
        raise AskjaError(rc, f"cannot load params file {path}")
    return rp.as_dict()


def _run_params(d: dict) -> RunParams:
    rp = RunParams()
    for k, _ in RunParams._fields_:
        if k == "n":
            for i, v in enumerate(d["n"]):
                rp.n[i] = int(v)
        elif k in d:
            setattr(rp, k, d[k])
    return rp


def params_store(infile: str, outfile: str, d: dict, timestep: int, taken: int):
    L = library()
    rp = _run_params(d)
    rc = L.askja_params_store(infile.encode(), outfile.encode(), ctypes.byref(rp), int(timestep), int(taken))
    if rc != ASKJA_OK:
        raise AskjaError(rc, f"cannot store params {infile} -> {outfile}")


def file_stem(d: dict, directory: str, kind: str) -> str:
    L = library()
    rp = _run_params(d)
    buf = ctypes.create_string_buffer(1024)
    rc = L.askja_file_stem(ctypes.byref(rp), directory.encode(), kind.encode(), buf, 1024)
    if rc != ASKJA_OK:
        raise AskjaError(rc, "file stem")
    return buf.value.decode()


def conf_write(path: str, conf: np.ndarray):
    L = library()
    a = np.ascontiguousarray(conf, dtype=np.complex128).view(np.float64)
    rc = L.askja_conf_write(path.encode(), _dptr(a), a.size)
    if rc != ASKJA_OK:
        raise AskjaError(rc, f"cannot write {path}")


def conf_read(path: str, shape) -> np.ndarray:
    L = library()
    out = np.empty(shape, np.complex128)
    a = out.view(np.float64)
    rc = L.askja_conf_read(path.encode(), _dptr(a), a.size)
    if rc != ASKJA_OK:
        raise AskjaError(rc, f"cannot read {path}")
    return out


@dataclass
class PinnedBuffer:
    """Page-locked host buffer from askja_host_alloc (cudaMallocHost)."""
    ptr: int
    nbytes: int

    @classmethod
    def alloc(cls, nbytes: int) -> "PinnedBuffer":
        p = library().askja_host_alloc(int(nbytes))
        if not p:
            raise AskjaError(-2, "askja_host_alloc failed")
        return cls(int(p), int(nbytes))

    def array(self, dtype, shape):
        buf = (ctypes.c_char * self.nbytes).from_address(self.ptr)
        return np.frombuffer(buf, dtype=dtype).reshape(shape)

    def free(self):
        if self.ptr:
            library().askja_host_free(ctypes.c_void_p(self.ptr))
            self.ptr = 0


class ChainParams(ctypes.Structure):
    _fields_ = [("nc", ctypes.c_int), ("dim", ctypes.c_int), ("n", ctypes.c_int * MAX_DIM),
                ("beta", ctypes.c_double), ("dt", ctypes.c_double), ("level", ctypes.c_int),
                ("seed", ctypes.c_uint64)]


class Batch:
    """Many independent chains of uneven shape advanced together
    (askja_batch_* of include/askja_gpu.h).  `chains` is a list of dicts with
    keys nc, dims, beta, dt, level, seed."""

    def __init__(self, chains, precision: str = "fp32", device: int = 0):
        L = library()
        vp = ctypes.c_void_p
        L.askja_batch_create.argtypes = [ctypes.POINTER(ChainParams), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(vp)]
        L.askja_batch_destroy.argtypes = [vp]
        L.askja_batch_destroy.restype = None
        L.askja_batch_last_error.argtypes = [vp]
        L.askja_batch_last_error.restype = ctypes.c_char_p
        L.askja_batch_stream.argtypes = [vp]
        L.askja_batch_stream.restype = vp
        L.askja_batch_hot_start.argtypes = [vp, ctypes.c_uint64]
        L.askja_batch_set_links.argtypes = [vp, ctypes.c_int, vp]
        L.askja_batch_get_links.argtypes = [vp, ctypes.c_int, vp]
        L.askja_batch_run.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(TrajResult)]
        L.askja_batch_plaquette.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        self.lib = L
        self.chains = [dict(c) for c in chains]
        arr = (ChainParams * len(chains))()
        for i, c in enumerate(self.chains):
            arr[i].nc, arr[i].dim = int(c["nc"]), len(c["dims"])
            for k, d in enumerate(c["dims"]):
                arr[i].n[k] = int(d)
            arr[i].beta, arr[i].dt = float(c["beta"]), float(c["dt"])
            arr[i].level, arr[i].seed = int(c.get("level", 8)), int(c.get("seed", 1 + i))
        self._b = ctypes.c_void_p()
        rc = L.askja_batch_create(arr, len(chains), {"fp64": FP64, "fp32": FP32}[precision], int(device),
                                  ctypes.byref(self._b))
        if rc != ASKJA_OK:
            raise AskjaError(rc, L.askja_batch_last_error(None).decode())

    def _ck(self, rc):
        if rc != ASKJA_OK:
            raise AskjaError(rc, self.lib.askja_batch_last_error(self._b).decode())

    def shape(self, c):
        if not 0 <= c < len(self.chains):
            raise AskjaError(-1, f"chain {c} out of range")
        ch = self.chains[c]
        return (int(np.prod(ch["dims"])), len(ch["dims"]), ch["nc"], ch["nc"])

    def close(self):
        if self._b:
            self.lib.askja_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream_ptr(self) -> int:
        return int(self.lib.askja_batch_stream(self._b) or 0)

    def hot_start(self, seed: int):
        self._ck(self.lib.askja_batch_hot_start(self._b, int(seed)))

    def set_links(self, c: int, u):
        u = np.ascontiguousarray(u, dtype=np.complex128).reshape(self.shape(c))
        self._ck(self.lib.askja_batch_set_links(self._b, int(c), u.ctypes.data))

    def get_links(self, c: int):
        out = np.empty(self.shape(c), np.complex128)
        self._ck(self.lib.askja_batch_get_links(self._b, int(c), out.ctypes.data))
        return out

    def run(self, ntraj: int, nsteps: int, use_graph: bool = True):
        res = (TrajResult * len(self.chains))()
        self._ck(self.lib.askja_batch_run(self._b, int(ntraj), int(nsteps), int(bool(use_graph)), res))
        return [r.as_dict() for r in res]

    def plaquette(self):
        out = (ctypes.c_double * len(self.chains))()
        self._ck(self.lib.askja_batch_plaquette(self._b, out))
        return list(out)


class Tuning(ctypes.Structure):
    _fields_ = [("path", ctypes.c_int), ("groups", ctypes.c_int), ("occupancy", ctypes.c_int),
                ("ncand", ctypes.c_int), ("best_us", ctypes.c_double), ("cand_path", ctypes.c_int * 24),
                ("cand_groups", ctypes.c_int * 24), ("cand_occ", ctypes.c_int * 24), ("cand_us", ctypes.c_double * 24)]

    def as_dict(self):
        n = self.ncand
        return {"path": self.path, "groups": self.groups, "occupancy": self.occupancy, "best_us": self.best_us,
                "candidates": [{"path": self.cand_path[i], "groups": self.cand_groups[i],
                                "occupancy": self.cand_occ[i], "us": self.cand_us[i]} for i in range(n)]}


def autotune(engine: "Engine", reps: int = 5) -> dict:
    """askja_autotune: time the kernel mappings for this engine's (NC, DIM,
    precision) and switch to the fastest (remembered for later engines)."""
    L = engine.lib
    L.askja_autotune.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(Tuning)]
    t = Tuning()
    engine._ck(L.askja_autotune(engine._ctx, int(reps), ctypes.byref(t)))
    return t.as_dict()


def set_tuning(engine: "Engine", d: dict):
    L = engine.lib
    L.askja_set_tuning.argtypes = [ctypes.c_void_p, ctypes.POINTER(Tuning)]
    t = Tuning()
    t.path, t.groups, t.occupancy = int(d["path"]), int(d.get("groups", 0)), int(d.get("occupancy", 0))
    engine._ck(L.askja_set_tuning(engine._ctx, ctypes.byref(t)))
