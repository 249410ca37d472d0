"""Build the askja B200 engine in-tree.

Produces
  askja_b200/libaskja_b200.so   the C-ABI library (include/askja_gpu.h)
  askja_b200/askja              the command-line driver (drop-in for ./askja)
  askja_b200/measure4d          the measurement driver (drop-in for ./measure4d)

CUDA sources are compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``); the CUDA runtime is linked
statically so the library does not depend on any Python package.
Run ``python -m askja_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libaskja_b200.so")
EXE = os.path.join(HERE, "askja")
MEASURE = os.path.join(HERE, "measure4d")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
# the image exports CXX pointing at a wrapper without OpenMP specs; the system g++ is used
CXX = "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
                  "--expt-relaxed-constexpr", "-ccbin", CXX]
CU_SOURCES = ["kernels_fp64.cu", "kernels_fp32.cu", "kernels_split.cu", "engine.cu", "static_plaq.cu", "batch.cu"]
# bench-only helper (compute-pipe peak probe for the roofline), not part of the product ABI
PEAK_SRC = "peak.cu"
PEAK_LIB = os.path.join(HERE, "libaskja_peak.so")
CPP_SOURCES = ["hostio.cpp"]
HEADERS = ["common.cuh", "small.cuh", "rows.cuh", "misc.cuh", "kernels.cuh", "launch.h", "batch.cuh", "tc.cuh", "eig.cuh", "pair.cuh", "tab.cuh", "split.cuh", "split.h"]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    header_deps = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "askja_gpu.h")]
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if _newer(o, [s] + header_deps):
            cmd = [NVCC] + NVFLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", s, "-o", o]
            jobs.append((cmd, o))
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if _newer(o, [s] + header_deps):
            jobs.append(([CXX, "-O2", "-fPIC", "-std=c++17", "-fvisibility=hidden", "-c", s, "-o", o], o))
    procs = []
    for cmd, o in jobs:
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True), cmd, o))
    failed = []
    for p, cmd, o in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((cmd, out))
            if os.path.exists(o):
                os.remove(o)
        elif out and (verbose or ptxas_info):
            print(out)
    if failed:
        for cmd, out in failed:
            sys.stderr.write(" ".join(cmd) + "\n" + out + "\n")
        raise RuntimeError("askja_b200 build failed")
    if _newer(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-ccbin", CXX, "-o", LIB] + objs + ["-cudart", "static"]
        subprocess.check_call(cmd)
    peak_src = os.path.join(CSRC, PEAK_SRC)
    if _newer(PEAK_LIB, [peak_src]):
        subprocess.check_call([NVCC] + NVFLAGS + ["-shared", peak_src, "-o", PEAK_LIB, "-cudart", "static"])
    libdir = os.path.dirname(LIB)
    for src, exe in (("askja_main.cpp", EXE), ("measure4d_main.cpp", MEASURE)):
        main_src = os.path.join(CSRC, src)
        if _newer(exe, [main_src, LIB, os.path.join(ROOT, "include", "askja_gpu.h")]):
            subprocess.check_call([CXX, "-O2", "-std=c++17", main_src, "-o", exe, "-L" + libdir, "-laskja_b200",
                                   "-Wl,-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
