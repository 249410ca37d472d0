"""askja_plaqexp_static, the allocation-free entry point, against the
existing askja_PlaqExp on the same links.

It serves callers that cannot let a library allocate GPU memory (device memory
owned by their own pool allocator, or a fixed memory budget where a cudaMalloc
would fail or stall the device), so here the caller's memory comes from torch
and the entry point is called through the C ABI with raw device pointers.
This file is named so that pytest collects it last."""
import ctypes

import numpy as np
import pytest

import askja_b200 as ab

pytestmark = pytest.mark.gpu


def _soa(u: np.ndarray, precision: str) -> np.ndarray:
    """U-conf (V, D, N, N) -> the plain structure-of-arrays order [d][r][c][site]."""
    a = np.ascontiguousarray(np.transpose(u, (1, 2, 3, 0)))
    return a.astype(np.complex64 if precision == "fp32" else np.complex128)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("nc,dims", [(3, [6, 4, 4, 5]), (2, [8, 3, 5]), (5, [3, 3, 2, 2])])
def test_static_plaqexp_matches_plaqexp(precision, nc, dims):
    import torch

    lib = ab.library()
    lib.askja_plaqexp_static.argtypes = [ctypes.POINTER(ab.Params), ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p]
    lib.askja_plaqexp_static.restype = ctypes.c_int
    # the entry point reads plain FP32 links, so its FP32 counterpart is an
    # engine holding exactly those (the FP32-only storage, no residual plane)
    engine_precision = "fp32-lean" if precision == "fp32" else precision
    with ab.Engine(nc, dims, beta=5.0, precision=engine_precision) as e:
        e.hot_start(11)
        want = np.array(e.PlaqExp())
        u = e.get_links()
        params = e.params
    params.precision = ab.FP32 if precision == "fp32" else ab.FP64  # the entry point's link storage
    links = torch.from_numpy(_soa(u, precision).view(np.float32 if precision == "fp32" else np.float64)).cuda()
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # the scratch array keeps the previous call's contents
        out.fill_(float("nan"))
        rc = lib.askja_plaqexp_static(ctypes.byref(params), links.data_ptr(), out.data_ptr(), stream)
        assert rc == 0, lib.askja_last_error(None)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12)


def test_static_plaqexp_rejects_oversized_volume():
    import torch

    lib = ab.library()
    lib.askja_plaqexp_static.argtypes = [ctypes.POINTER(ab.Params), ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p]
    p = ab.Params()
    p.nc, p.dim, p.precision, p.device = 3, 4, ab.FP32, 0
    for i in range(4):
        p.n[i] = 40  # 2,560,000 sites > 2,097,152
    dummy = torch.zeros(4, dtype=torch.float64, device="cuda")
    rc = lib.askja_plaqexp_static(ctypes.byref(p), dummy.data_ptr(), dummy.data_ptr(), None)
    assert rc == -1
    assert b"static scratch limit" in lib.askja_last_error(None)
