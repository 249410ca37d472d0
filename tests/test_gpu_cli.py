"""The askja CLI drop-in end to end: params file in, output-DIM<D>/ out,
resume from the master params, and the reference's own measure4d (compiled
from the reference sources against the GSL shim, where available) reading the
configurations we wrote, agreeing with the engine's own measurements."""
import os
import re
import subprocess

import numpy as np
import pytest

import askja_b200 as ab
from oracle import REF_DIR

pytestmark = pytest.mark.gpu

MEASURE4D = os.path.join(REF_DIR, "measure4d_ref")

PARAMS = """#Parameters_file
NC              {nc}
DIM             {dim}
{dims}BETA            {beta}
DT              {dt}
STEPS           {steps}
UPDATE          {update}
UPDATE2         {update2}
CONFTAKE        {conftake}
LEVEL           {level}
VERBOSE         0
RUNCONTINUE     0
RANDOM          0
"""


def write_params(path, nc, n, beta, dt, steps, update, update2, conftake, level):
    dims = "".join(f"N{i}              {v}\n" for i, v in enumerate(n))
    with open(path, "w") as f:
        f.write(PARAMS.format(nc=nc, dim=len(n), dims=dims, beta=beta, dt=dt, steps=steps, update=update,
                              update2=update2, conftake=conftake, level=level))


def run_askja(cwd, *args):
    r = subprocess.run([ab.EXE_PATH, *args], cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "Finished successfully" in r.stdout
    return r.stdout


@pytest.mark.parametrize("precision", ["--fp64", "--fp32"])
def test_cli_run_and_resume(tmp_path, precision):
    nc, n, beta, dt = 3, [4, 4, 4, 4], 5.7, 0.02
    write_params(tmp_path / "p.txt", nc, n, beta, dt, steps=60, update=5, update2=10, conftake=2, level=8)
    out = run_askja(tmp_path, precision, "p.txt")
    d = ab.params_load(str(tmp_path / "p.txt"))
    outdir = tmp_path / "output-DIM4"
    stem = lambda kind: os.path.basename(ab.file_stem(d, "output-DIM4", kind))
    cons = (outdir / (stem("constraints") + ".dat")).read_text().splitlines()
    wil = (outdir / (stem("Wilson") + ".dat")).read_text().splitlines()
    assert cons[0].startswith("#Time") and wil[0].startswith("#Time")
    assert len(cons) == 1 + 1 + 60 // 5 and len(wil) == len(cons)
    first = [float(x) for x in cons[1].split()]
    assert first[0] == 0.0 and abs(first[1]) < 1e-20 and first[4] == 0.0  # cold start: EM = 0, Gauss law ~ 0
    # 60 MD steps: trajectory ends at t = 10, 20, ..., 60 -> 6 trajectories, a conf every 2
    assert out.count("INFO: Final energy") == 6
    confs = sorted(p.name for p in outdir.glob("U-*.conf"))
    assert len(confs) == 3
    for c in confs:
        assert (outdir / c).stat().st_size == 256 * 4 * 9 * 16
    master = outdir / (stem("master") + ".params")
    m = ab.params_load(str(master))
    assert m["runcontinue"] == 1 and m["taken"] == 3 and m["start"] == 60 and m["ntot"] == 6
    # NACC is read back rounded down to a multiple of CONFTAKE (sun.cpp:904)
    assert m["nacc"] % 2 == 0 and m["nacc"] + m["nrec"] <= 6
    # stored configurations are SU(3)
    u = ab.conf_read(str(outdir / confs[-1]), (256, 4, 3, 3)).reshape(-1, 3, 3)
    assert np.abs(np.einsum("lij,lkj->lik", u, u.conj()) - np.eye(3)).max() < 1e-5
    # resume: the master file is a params file with the trailer
    run_askja(tmp_path, precision, str(master.relative_to(tmp_path)))
    m2 = ab.params_load(str(master))
    assert m2["taken"] == 6 and m2["start"] == 120 and m2["ntot"] == 12
    cons2 = (outdir / (stem("constraints") + ".dat")).read_text().splitlines()
    assert len(cons2) == len(cons) + 60 // 5  # appended, no new header, no t=0 line
    assert len(sorted(outdir.glob("U-*.conf"))) == 6


def test_cli_errors(tmp_path):
    r = subprocess.run([ab.EXE_PATH, "missing.txt"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode != 0 and "could not be opened" in r.stdout
    (tmp_path / "bad.txt").write_text("#x\nNC 3\nDIM 2\nN0 4\n")
    r = subprocess.run([ab.EXE_PATH, "bad.txt"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode != 0 and "malformed" in r.stdout


@pytest.mark.skipif(not os.path.exists(MEASURE4D), reason="shim-built reference measure4d not available")
def test_reference_measure4d_reads_our_output(tmp_path):
    nc, n, beta = 2, [4, 3, 3, 2], 2.4
    write_params(tmp_path / "p.txt", nc, n, beta, 0.05, steps=80, update=10, update2=10, conftake=1, level=8)
    run_askja(tmp_path, "p.txt")
    d = ab.params_load(str(tmp_path / "p.txt"))
    master = os.path.basename(ab.file_stem(d, "output-DIM4", "master")) + ".params"
    r = subprocess.run([MEASURE4D, os.path.join("output-DIM4", master)], cwd=tmp_path, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0 and "Finished successfully" in r.stdout, r.stdout[-2000:]
    rav = tmp_path / "rav-DIM4" / (os.path.basename(ab.file_stem(d, "rav-DIM4", "Nrav")) + ".dat")
    last = [float(x) for x in rav.read_text().splitlines()[-1].split()]
    taken = int(last[0])
    assert taken == 8
    # the same observables from our engine on the same files
    V = int(np.prod(n))
    vals = []
    with ab.Engine(nc, n, beta=beta) as e:
        for k in range(taken):
            path = tmp_path / "output-DIM4" / (os.path.basename(ab.file_stem(d, "output-DIM4", "U")) + f"-{k}.conf")
            e.set_links(ab.conf_read(str(path), (V, 4, nc, nc)))
            t, s = e.PlaqExp()
            vals.append((e.PolyakovLoop(), e.WilsonLoopDir(1), t * beta / n[0], s * beta / n[0]))
    vals = np.array(vals)
    mean = vals.mean(axis=0)
    err = np.sqrt(((vals - mean) ** 2).sum(axis=0)) / taken
    np.testing.assert_allclose([last[1], last[3], last[5], last[7]], mean, rtol=1e-5)
    np.testing.assert_allclose([last[2], last[4], last[6], last[8]], err, rtol=1e-4, atol=1e-6)
    assert (last[9], last[10], last[11]) == (n[0], n[1], beta)
