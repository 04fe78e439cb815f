"""Build libbv_b200.so in-tree: nvcc for sm_100a (CUDA sources), g++ for the
host layout code, linked into one shared library next to this file.

    python -m blockvecchia_b200.build          # incremental
    python -m blockvecchia_b200.build --clean  # from scratch
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbv_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("BV_CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
                  "--expt-relaxed-constexpr", "-I", INCLUDE]
CXXFLAGS = ["-O3", "-fPIC", "-fopenmp", "-std=c++17", "-I", INCLUDE]

CU_SOURCES = ["bv_llh.cu", "bv_knn.cu", "bv_llh_mixed.cu", "bv_server.cu"]
APPS = {"test_dvecchia_batch": os.path.join(HERE, "apps", "test_dvecchia_batch.cpp")}
BIN = os.path.join(HERE, "bin")
CPP_SOURCES = ["bv_layout.cpp"]
HEADERS = [f for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] if os.path.isdir(CSRC) else []


def _stale(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [src] + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "bv.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {cmd[-1]}")
    return r


def build(clean: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    if clean and os.path.isdir(BUILD):
        shutil.rmtree(BUILD)
    os.makedirs(BUILD, exist_ok=True)
    objs, jobs = [], []
    for s in CU_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        if _stale(obj, src) or ptxas_v:
            jobs.append([NVCC] + NVFLAGS + (["-Xptxas", "-v"] if ptxas_v else []) + ["-c", src, "-o", obj])
        objs.append(obj)
    for s in CPP_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        if _stale(obj, src):
            jobs.append([CXX] + CXXFLAGS + ["-c", src, "-o", obj])
        objs.append(obj)
    # The translation units compile independently: all at once.
    with ThreadPoolExecutor(max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for r in ex.map(_run, jobs):
            if verbose or ptxas_v:
                sys.stdout.write(r.stdout + r.stderr)
    changed = bool(jobs)
    if changed or not os.path.exists(LIB):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xcompiler", "-fopenmp", "-lgomp"])
        changed = True
    # Command-line driver with the reference's flags, linked against the library.
    os.makedirs(BIN, exist_ok=True)
    for name, src in APPS.items():
        exe = os.path.join(BIN, name)
        if changed or not os.path.exists(exe) or os.path.getmtime(src) > os.path.getmtime(exe):
            _run([CXX, "-O2", "-std=c++17", "-I", INCLUDE, src, "-o", exe, "-L", HERE, "-lbv_b200",
                  "-Wl,-rpath,$ORIGIN/.."])
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print registers/spills/smem per kernel")
    a = ap.parse_args()
    print(build(clean=a.clean, verbose=True, ptxas_v=a.ptxas_v))
