"""Ensemble parity against a run of the reference itself.

tests/golden/ensemble_su3_4x4x4x4.json holds what the reference's own askja
and measure4d produced for an SU(3) 4^4 chain (BETA 5.70, DT 0.02, LEVEL 8,
50 MD steps per trajectory, 16000 trajectories from a cold start; made by
tests/golden/gen_ensemble.py).  Here the GPU askja CLI runs the same params
file (with a configuration stored every 4th trajectory) in FP64 and in
FP32-mixed, the GPU measure4d measures its configurations after the same
number of thermalisation trajectories, and the ensemble averages of the plaquettes (temporal and
spatial, beta/N0 normalised as in the Nrav file) and of the Polyakov loop
must agree with the reference's within 2 sigma.  Sigma combines both chains'
errors of the mean from bins of 200 consecutive trajectories (the Nrav
errors of measure4d ignore the autocorrelation, which at this coupling --
near the N0 = 4 deconfinement transition -- is long for the Polyakov loop).  The two chains draw
different random numbers (the reference's GSL stream is not reproducible),
so this is a statistical comparison; the engine is deterministic for a fixed
seed (RANDOM 0), so the outcome is too."""
import json
import os
import subprocess

import numpy as np
import pytest

import askja_b200 as ab
from test_gpu_cli import run_askja, write_params

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ensemble_su3_4x4x4x4.json")
MEASURE4D = os.path.join(os.path.dirname(ab.LIB_PATH), "measure4d")
OBS = ("polyakov", "plaq_t", "plaq_s")
CONFTAKE = 4  # GPU chains: a configuration every 4th trajectory


def binned(values, size):
    v = np.asarray(values, dtype=np.float64)
    nb = len(v) // size
    b = v[:nb * size].reshape(nb, size).mean(axis=1)
    return float(b.mean()), float(b.std(ddof=1) / np.sqrt(nb))


@pytest.mark.parametrize("precision", ["--fp64", "--fp32"])
def test_ensemble_matches_reference_run(tmp_path, precision):
    fx = json.load(open(FIXTURE))
    p = fx["params"]
    nc, dims, beta = p["nc"], p["dims"], p["beta"]
    ntraj = p["trajectories"]
    skip, size = fx["skip"] // CONFTAKE, fx["bin"] // CONFTAKE  # in stored configurations
    write_params(tmp_path / "p.txt", nc, dims, f"{beta:.2f}", p["dt"], steps=ntraj * p["update2"],
                 update=p["update2"], update2=p["update2"], conftake=CONFTAKE, level=p["level"])
    run_askja(tmp_path, precision, "p.txt")
    d = ab.params_load(str(tmp_path / "p.txt"))
    master = os.path.join("output-DIM4", os.path.basename(ab.file_stem(d, "output-DIM4", "master")) + ".params")
    r = subprocess.run([MEASURE4D, master, str(skip)], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "Finished successfully" in r.stdout, r.stdout[-2000:]
    rav = tmp_path / "rav-DIM4" / (os.path.basename(ab.file_stem(d, "rav-DIM4", "Nrav")) + ".dat")
    nrav = [float(x) for x in rav.read_text().splitlines()[-1].split()]
    taken = int(nrav[0])
    assert taken == ntraj // CONFTAKE
    # per-configuration values for the binned errors, from the engine on the stored files
    V = int(np.prod(dims))
    series = {k: [] for k in OBS}
    u_stem = os.path.basename(ab.file_stem(d, "output-DIM4", "U"))
    with ab.Engine(nc, dims, beta=beta) as e:
        for k in range(skip, taken):
            e.set_links(ab.conf_read(str(tmp_path / "output-DIM4" / f"{u_stem}-{k}.conf"), (V, len(dims), nc, nc)))
            t, s = e.PlaqExp()
            series["polyakov"].append(e.PolyakovLoop())
            series["plaq_t"].append(t * beta / dims[0])
            series["plaq_s"].append(s * beta / dims[0])
    # measure4d's own averages are those of the same configurations
    np.testing.assert_allclose([nrav[1], nrav[5], nrav[7]], [np.mean(series[k]) for k in OBS], rtol=1e-5)
    report = {}
    for k in OBS:
        m_gpu, e_gpu = binned(series[k], size)
        b = np.asarray(fx["bins"][k])
        m_ref, e_ref = float(b.mean()), float(b.std(ddof=1) / np.sqrt(len(b)))
        sigma = float(np.hypot(e_gpu, e_ref))
        report[k] = (m_gpu, e_gpu, m_ref, e_ref, abs(m_gpu - m_ref) / sigma)
    msg = "; ".join(f"{k}: GPU {m:.6f}({e:.6f}) vs reference {mr:.6f}({er:.6f}), {z:.2f} sigma"
                    for k, (m, e, mr, er, z) in report.items())
    print(msg)
    assert all(v[4] <= 2.0 for v in report.values()), msg
    # the reference's Nrav line is the mean of the same configurations the bins were made from
    for k, j in (("polyakov", "polyakov"), ("plaq_t", "plaq_t"), ("plaq_s", "plaq_s")):
        nb = len(fx["bins"][k]) * size
        if nb == fx["taken"] - skip:
            assert np.mean(fx["bins"][k]) == pytest.approx(fx["nrav"][j], rel=1e-5)  # Nrav: 6 digits
