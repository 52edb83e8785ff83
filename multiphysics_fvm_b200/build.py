"""Build libfvm_b200.so (sm_100a) in-tree from multiphysics_fvm_b200/csrc/*.cu.

    python -m multiphysics_fvm_b200.build [-j N] [--force]

Each translation unit is compiled separately (in parallel) with
``nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3``.  Units that hold
float64 kernels or float64 reductions (``*_double*.cu``, ``fvm_api.cu``) are
compiled with ``--fmad=false`` so that the float64 build rounds every operation
like NumPy does; the float32 kernels keep FMA contraction.  Objects go to
``csrc/build/``; the shared library is written next to this file.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(CSRC, "build")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "libfvm_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libfvm_b200")


def _flags(src: str) -> list[str]:
    f = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
                "-I", CSRC, "-I", INCLUDE]
    base = os.path.basename(src)
    if "_double" in base or base == "fvm_api.cu":
        f += ["--fmad=false"]
    return f


def _deps() -> float:
    newest = 0.0
    for d in (CSRC, INCLUDE):
        for fn in os.listdir(d):
            if fn.endswith((".cuh", ".h")):
                newest = max(newest, os.path.getmtime(os.path.join(d, fn)))
    return newest


def _compile(nvcc: str, src: str, force: bool, hdr_time: float) -> str:
    obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
    if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
            and os.path.getmtime(obj) >= hdr_time):
        return obj
    cmd = [nvcc] + _flags(src) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
    return obj


def build(jobs: int | None = None, force: bool = False, verbose: bool = False) -> str:
    nvcc = nvcc_path()
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))
    hdr = _deps()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(nvcc, s, force, hdr), srcs))
    if (force or not os.path.exists(LIB)
            or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs)):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcuda"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
        if verbose:
            print(f"linked {LIB}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.j, a.force, verbose=True))
    sys.exit(0)
