import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")
GOLDEN = sorted(glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def load_golden(path):
    with np.load(path) as z:
        d = {k: z[k] for k in z.files}
    for k in ("nc", "level", "lf_steps"):
        d[k] = int(d[k])
    for k in ("beta", "eps_e", "eps_u"):
        d[k] = float(d[k])
    d["dims"] = [int(x) for x in d["dims"]]
    d["name"] = os.path.basename(path)[:-4]
    return d


@pytest.fixture(params=GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def golden(request):
    return load_golden(request.param)


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)
