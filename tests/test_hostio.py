"""Host-side parts of the drop-in (no GPU): the C-ABI library loads and
exports every entry point include/askja_gpu.h declares; the params file,
master params, file stems and U-conf files are byte-compatible with the
reference (checked against the shim-built reference askja where available);
error paths return status codes; the engine refuses to run without a GPU."""
import os
import re
import subprocess

import numpy as np
import pytest

import askja_b200 as ab
from oracle import REF_DIR

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ASKJA_REF = os.path.join(REF_DIR, "askja_ref")

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


def write_params(path, nc=3, n=(4, 4, 4, 4), beta=5.70, dt=0.02, steps=40, update=10, update2=10, conftake=2,
                 level=8):
    dims = "".join(f"N{i}              {v}\n" for i, v in enumerate(n))
    with open(path, "w") as f:
        f.write(PARAMS.format(nc=nc, dim=len(n), dims=dims, beta=beta, dt=dt, steps=steps, update=update,
                              update2=update2, conftake=conftake, level=level))


def test_library_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "askja_gpu.h")).read()
    declared = sorted(set(re.findall(r"ASKJA_API\s+[\w\s\*]+?\b(askja_\w+)\(", hdr)))
    assert sorted(ab.EXPORTS) == declared
    lib = ab.library()
    for name in declared:
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", ab.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (askja_\w+)", out))
    assert set(declared) <= exported


def test_version_and_kernels_are_sm100a():
    assert b"sm_100a" in ab.library().askja_version()


def test_no_cpu_fallback():
    """Without a CUDA device askja_create fails loudly."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(ab.AskjaError) as e:
        ab.Engine(3, [4, 4], beta=5.7)
    assert e.value.code in (-5, -2)


def test_params_load(tmp_path):
    p = tmp_path / "p.txt"
    write_params(p, nc=8, n=(10, 10, 1, 1, 1, 1, 1, 1, 1, 1), beta=20000, dt=0.01, steps=100000, update=500,
                 update2=1000, conftake=10, level=8)
    d = ab.params_load(str(p))
    assert d["nc"] == 8 and d["dim"] == 10 and d["n"] == [10, 10] + [1] * 8
    assert d["beta"] == 20000 and d["dt"] == 0.01 and d["steps"] == 100000
    assert (d["update"], d["update2"], d["conftake"], d["level"]) == (500, 1000, 10, 8)
    assert d["runcontinue"] == 0 and d["start"] == 1


def test_params_errors(tmp_path):
    with pytest.raises(ab.AskjaError) as e:
        ab.params_load(str(tmp_path / "missing.txt"))
    assert e.value.code == -3
    bad = tmp_path / "bad.txt"
    bad.write_text("#Parameters_file\nNC 3\nDIM 4\nN0 4\n")
    with pytest.raises(ab.AskjaError) as e:
        ab.params_load(str(bad))
    assert e.value.code == -6


def test_resume_trailer_roundtrip(tmp_path):
    p = tmp_path / "p.txt"
    write_params(p, conftake=4)
    d = ab.params_load(str(p))
    d.update(nacc=7, nac1=3, nrec=2, ntot=9)
    m = tmp_path / "master.params"
    ab.params_store(str(p), str(m), d, 90, 2)
    r = ab.params_load(str(m))
    assert r["runcontinue"] == 1 and r["start"] == 90 and r["taken"] == 2
    assert r["nacc"] == 4  # NACC rounded down to a multiple of CONFTAKE (sun.cpp:904)
    assert (r["nac1"], r["nrec"], r["ntot"]) == (3, 2, 9)


def test_conf_roundtrip_and_short_file(tmp_path):
    x = (np.random.default_rng(0).standard_normal((6, 2, 3, 3)) + 1j).astype(np.complex128)
    f = tmp_path / "U.conf"
    ab.conf_write(str(f), x)
    assert f.stat().st_size == x.size * 16
    np.testing.assert_array_equal(ab.conf_read(str(f), x.shape), x)
    # the layout is the raw doubles, (re, im) interleaved, no header
    np.testing.assert_array_equal(np.fromfile(f, dtype=np.float64), x.view(np.float64).ravel())
    with pytest.raises(ab.AskjaError):
        ab.conf_read(str(f), (7, 2, 3, 3))
    with pytest.raises(ab.AskjaError):
        ab.conf_read(str(tmp_path / "none.conf"), x.shape)
    with pytest.raises(ab.AskjaError):
        ab.conf_write(str(tmp_path / "nodir" / "x.conf"), x)


@pytest.mark.skipif(not os.path.exists(ASKJA_REF), reason="shim-built reference askja not available")
def test_master_params_and_stems_match_reference(tmp_path):
    """Run the reference askja (shim build) and check that our store_parameters
    and file stems reproduce its master file and file names byte for byte."""
    ref = tmp_path / "ref"
    ref.mkdir()
    write_params(ref / "p.txt", nc=2, n=(4, 3, 2), beta=2.5, dt=0.05, steps=20, update=5, update2=5, conftake=2,
                 level=6)
    subprocess.run([ASKJA_REF, "p.txt"], cwd=ref, check=True, capture_output=True, env={**os.environ,
                                                                                        "OMP_NUM_THREADS": "1"})
    outdir = ref / "output-DIM3"
    names = sorted(os.listdir(outdir))
    d = ab.params_load(str(ref / "p.txt"))
    stem = os.path.basename(ab.file_stem(d, "output-DIM3", "constraints"))
    assert stem + ".dat" in names
    assert os.path.basename(ab.file_stem(d, "output-DIM3", "U")) + "-0.conf" in names
    master = [n for n in names if n.startswith("master")][0]
    assert os.path.basename(ab.file_stem(d, "output-DIM3", "master")) + ".params" == master
    ref_master = (outdir / master).read_text()
    m = ab.params_load(str(outdir / master))
    ours = tmp_path / "ours.params"
    d.update(nacc=m["nacc"], nac1=m["nac1"], nrec=m["nrec"], ntot=m["ntot"])
    ab.params_store(str(ref / "p.txt"), str(ours), d, m["start"], m["taken"])
    assert ours.read_text() == ref_master
    # U-conf size: V * DIM * NC^2 complex doubles
    conf = outdir / [n for n in names if n.endswith("-0.conf")][0]
    assert conf.stat().st_size == 4 * 3 * 2 * 3 * 2 * 2 * 16
