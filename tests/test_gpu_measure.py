"""The measurement side of the drop-in: the line eigenphases of getevs
(measurements4d.cpp:185-309) on the GPU against an independent numpy
restatement, and the measure4d driver against the reference's own measure4d
(compiled from the reference sources against the GSL shim) on the same askja
output directory.

Tolerances: eigenphases 1e-9 absolute in FP64 (Hessenberg + shifted QR in
FP64 against LAPACK), 1e-5 on FP32-stored links; the rav/W24/P5corr files
agree field by field to 1e-9 relative (both print six significant digits of
FP64 sums taken in a different order)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import askja_b200 as ab
from oracle import REF_DIR, Oracle, fields
from test_gpu_cli import run_askja, write_params

pytestmark = pytest.mark.gpu

MEASURE4D_REF = os.path.join(REF_DIR, "measure4d_ref")
MEASURE4D = os.path.join(os.path.dirname(ab.LIB_PATH), "measure4d")


def line(u, O, start, d, extent):
    pos, W = start, u[start, d].copy()
    for _ in range(extent - 1):
        pos = O.getplus(pos, d)
        W = W @ u[pos, d]
    return W


def sorted_phases(W, nc):
    ph = np.angle(np.linalg.eigvals(W))
    wind = ph.sum() / (2 * np.pi)
    if wind > 0.1 or wind < -0.1:
        ph = ph - wind * 2 * np.pi / nc
    return np.sort(ph)


def getevs(u, dims, nc):
    """measurements4d.cpp:185-309 restated: averaged sorted eigenphases of the
    Wilson lines along 1 through (x0,0,..) and the Polyakov lines along 0
    through (0,x1,0,..)."""
    O = Oracle(nc, dims)
    stride = [int(np.prod(dims[i + 1:])) for i in range(len(dims))]
    w = np.mean([sorted_phases(line(u, O, x0 * stride[0], 1, dims[1]), nc) for x0 in range(dims[0])], axis=0)
    p = np.mean([sorted_phases(line(u, O, x1 * stride[1], 0, dims[0]), nc) for x1 in range(dims[1])], axis=0)
    return w, p


CASES = [(2, [4, 3, 2, 2]), (3, [4, 3, 2, 2]), (5, [3, 4, 2]), (8, [3, 4]), (16, [2, 3, 2]), (32, [3, 2]),
         (64, [2, 2])]


@pytest.mark.parametrize("nc,dims", CASES, ids=[f"su{n}_{'x'.join(map(str, d))}" for n, d in CASES])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_eigenphases_vs_numpy(nc, dims, precision):
    rng = np.random.default_rng(nc * 13 + len(dims))
    V = int(np.prod(dims))
    u = fields.haar(nc, V * len(dims), rng).reshape(V, len(dims), nc, nc)
    if precision == "fp32":
        u = u.astype(np.complex64).astype(np.complex128)
    want_w, want_p = getevs(u, dims, nc)
    with ab.Engine(nc, dims, beta=1.0, precision=precision) as e:
        e.set_links(u)
        w, p = e.eigenphases()
    tol = 1e-9 if precision == "fp64" else 1e-5
    np.testing.assert_allclose(w, want_w, atol=tol)
    np.testing.assert_allclose(p, want_p, atol=tol)


def test_eigenphases_cold_start():
    """Unit lines: every phase 0."""
    with ab.Engine(4, [3, 3, 2], beta=1.0) as e:
        e.initializeU()
        w, p = e.eigenphases()
    np.testing.assert_allclose(w, 0.0, atol=1e-14)
    np.testing.assert_allclose(p, 0.0, atol=1e-14)


def read_table(path):
    rows = []
    for ln in open(path).read().splitlines():
        if ln.startswith("#"):
            rows.append(ln.split())
        else:
            rows.append([float(x) for x in ln.split()])
    return rows


def assert_tables_close(a, b):
    assert len(a) == len(b)
    for ra, rb in zip(a, b):
        assert len(ra) == len(rb)
        for x, y in zip(ra, rb):
            if isinstance(x, str):
                assert x == y
            else:
                assert x == pytest.approx(y, rel=1e-9, abs=1e-12)


@pytest.mark.skipif(not os.path.exists(MEASURE4D_REF), reason="shim-built reference measure4d not available")
@pytest.mark.parametrize("nc,n", [(2, [4, 3, 3, 2]), (3, [6, 4, 4, 4])])
def test_measure4d_matches_reference(tmp_path, nc, n):
    beta = 2.4 if nc == 2 else 5.7
    write_params(tmp_path / "p.txt", nc, n, beta, 0.05, steps=90, update=10, update2=10, conftake=1, level=8)
    run_askja(tmp_path, "p.txt")
    d = ab.params_load(str(tmp_path / "p.txt"))
    master = os.path.join("output-DIM4", os.path.basename(ab.file_stem(d, "output-DIM4", "master")) + ".params")
    skip = 2
    r = subprocess.run([MEASURE4D_REF, master, str(skip), "0", "0"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0 and "Finished successfully" in r.stdout, r.stdout[-2000:]
    shutil.move(str(tmp_path / "rav-DIM4"), str(tmp_path / "rav-ref"))
    r = subprocess.run([MEASURE4D, master, str(skip), "0", "0"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0 and "Finished successfully" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
    for kind in ("Nrav", "W24", "P5corr"):
        name = os.path.basename(ab.file_stem(d, "x", kind)) + ".dat"
        assert_tables_close(read_table(tmp_path / "rav-DIM4" / name), read_table(tmp_path / "rav-ref" / name))


def test_measure4d_eigenphase_histogram(tmp_path):
    """GET_EV_DIST = 1: the Hist file against the histogram of the numpy
    eigenphases of every configuration (the reference's binning)."""
    nc, n, beta = 3, [4, 3, 3, 2], 5.0
    write_params(tmp_path / "p.txt", nc, n, beta, 0.05, steps=60, update=10, update2=10, conftake=1, level=8)
    run_askja(tmp_path, "p.txt")
    d = ab.params_load(str(tmp_path / "p.txt"))
    master = os.path.join("output-DIM4", os.path.basename(ab.file_stem(d, "output-DIM4", "master")) + ".params")
    r = subprocess.run([MEASURE4D, master, "0", "0", "1"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "Finished successfully" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
    taken = ab.params_load(str(tmp_path / master))["taken"]
    assert taken >= 4
    width = np.pi / (2 * nc)
    bins = int(np.floor(2 * np.pi / width))
    wh, ph = np.zeros(bins), np.zeros(bins)
    V = int(np.prod(n))
    for k in range(taken):
        path = tmp_path / "output-DIM4" / (os.path.basename(ab.file_stem(d, "output-DIM4", "U")) + f"-{k}.conf")
        u = ab.conf_read(str(path), (V, 4, nc, nc))
        w, p = getevs(u, n, nc)
        for x, h in ((w, wh), (p, ph)):
            for v in x:
                h[int(np.floor((v + np.pi) / width))] += 1
    hist = np.array(read_table(tmp_path / "rav-DIM4" / (os.path.basename(ab.file_stem(d, "x", "Hist")) + ".dat")))
    assert hist.shape == (bins, 3)
    np.testing.assert_allclose(hist[:, 0], -np.pi + (np.arange(bins) + 0.5) * width, rtol=1e-5)
    np.testing.assert_allclose(hist[:, 1], ph / taken, atol=1e-6)
    np.testing.assert_allclose(hist[:, 2], wh / taken, atol=1e-6)
