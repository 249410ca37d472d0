"""Generate the ensemble fixture tests/golden/ensemble_su3_4x4x4x4.json from a
run of the reference itself.

The reference's own askja (sun.cpp compiled unchanged against the project's
GSL shim by oracle/Makefile, as oracle/_ref/askja_ref_clock: its time() is a
counter that advances on every call) runs an SU(3) 4^4 HMC chain from a cold
start: BETA 5.70, DT 0.02, LEVEL 8, UPDATE2 50 (50 MD steps per trajectory),
16000 trajectories, a configuration stored after every trajectory.  The
reference reseeds its generator from time(NULL) for every momentum refresh and
every Metropolis uniform (sun.cpp:1268-1311); with the wall clock, the ~20
trajectories it runs per second here would share seeds -- the same momenta and
uniforms -- and the chain would sample a biased ensemble (a first fixture made
that way had a Polyakov loop 2-4 sigma below two independent GPU runs).  The reference's own measure4d (oracle/_ref/measure4d_ref) then
measures the stored configurations after SKIP thermalisation ones and writes
its Nrav line (<|P|>, <W>, beta/N0 <plaquette> temporal and spatial, each with
the reference's naive error).  The same per-configuration observables are
taken with the reference's measurement routines (libref_measure4d.so) and
stored as means over bins of BIN consecutive configurations, from which the
test forms errors that include the autocorrelation.

Needs oracle/_ref (built where the reference sources are); never runs on the
GPU host.  Takes about half an hour on 8 cores.

    python tests/golden/gen_ensemble.py
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import REF_DIR, Reference  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ensemble_su3_4x4x4x4.json")

NC, DIMS, BETA, DT, LEVEL, UPDATE2 = 3, [4, 4, 4, 4], 5.70, 0.02, 8, 50
NTRAJ, SKIP, BIN = 16000, 400, 200

PARAMS = """#Parameters_file
NC              {nc}
DIM             {dim}
{dims}BETA            {beta:.2f}
DT              {dt}
STEPS           {steps}
UPDATE          {update2}
UPDATE2         {update2}
CONFTAKE        1
LEVEL           {level}
VERBOSE         0
RUNCONTINUE     0
RANDOM          0
"""


def params_text(ntraj: int) -> str:
    dims = "".join(f"N{i}              {v}\n" for i, v in enumerate(DIMS))
    return PARAMS.format(nc=NC, dim=len(DIMS), dims=dims, beta=BETA, dt=DT, steps=ntraj * UPDATE2, update2=UPDATE2,
                         level=LEVEL)


def stem() -> str:
    # sun.cpp:1124 file stem
    return f"N{NC}-Nt{DIMS[0]}-Ns{DIMS[1]}-BETA{BETA:.2f}-DT{DT:.4f}-U{UPDATE2 * DT:.4f}-CT1"


def main():
    work = tempfile.mkdtemp(prefix="askja_ens_")
    with open(os.path.join(work, "p.txt"), "w") as f:
        f.write(params_text(NTRAJ))
    env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1))
    r = subprocess.run([os.path.join(REF_DIR, "askja_ref_clock"), "p.txt"], cwd=work, env=env, capture_output=True,
                       text=True)
    assert r.returncode == 0 and "Finished successfully" in r.stdout, r.stdout[-2000:]
    acc_line = [ln for ln in r.stdout.splitlines() if "Statistics" in ln][-1]
    master = os.path.join("output-DIM4", f"master-{stem()}.params")
    r = subprocess.run([os.path.join(REF_DIR, "measure4d_ref"), master, str(SKIP)], cwd=work, env=env,
                       capture_output=True, text=True)
    assert r.returncode == 0 and "Finished successfully" in r.stdout, r.stdout[-2000:]
    nrav = open(os.path.join(work, "rav-DIM4", f"Nrav-{stem()}.dat")).read().splitlines()[-1].split()
    taken = int(nrav[0])
    # per-configuration observables with the reference's measurement routines
    R = Reference(NC, DIMS, beta=BETA, level=LEVEL)
    V = int(np.prod(DIMS))
    series = {"polyakov": [], "wilson": [], "plaq_t": [], "plaq_s": []}
    for k in range(SKIP, taken):
        u = np.fromfile(os.path.join(work, "output-DIM4", f"U-{stem()}-{k}.conf"), dtype=np.float64)
        R.set("u", u.view(np.complex128).reshape(V, len(DIMS), NC, NC))
        t, s = R.PlaqExp()
        series["polyakov"].append(R.PolyakovLoop())
        series["wilson"].append(R.WilsonLoopDir(1))
        series["plaq_t"].append(t * BETA / DIMS[0])
        series["plaq_s"].append(s * BETA / DIMS[0])
    nb = (taken - SKIP) // BIN
    bins = {k: np.asarray(v[:nb * BIN]).reshape(nb, BIN).mean(axis=1).tolist() for k, v in series.items()}
    fixture = {
        "generator": "tests/golden/gen_ensemble.py: oracle/_ref/askja_ref_clock + oracle/_ref/measure4d_ref",
        "params": {"nc": NC, "dims": DIMS, "beta": BETA, "dt": DT, "level": LEVEL, "update2": UPDATE2,
                   "trajectories": NTRAJ, "conftake": 1, "random": 0},
        "reference_acceptance": acc_line.strip(),
        "skip": SKIP,
        "taken": taken,
        "nrav": {"taken": taken, "polyakov": float(nrav[1]), "polyakov_err": float(nrav[2]),
                 "wilson": float(nrav[3]), "wilson_err": float(nrav[4]), "plaq_t": float(nrav[5]),
                 "plaq_t_err": float(nrav[6]), "plaq_s": float(nrav[7]), "plaq_s_err": float(nrav[8])},
        "bin": BIN,
        "bins": bins,
    }
    with open(OUT, "w") as f:
        json.dump(fixture, f, indent=1)
    print(json.dumps(fixture["nrav"]))


if __name__ == "__main__":
    main()
