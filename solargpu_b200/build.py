"""Builds libsolargpu_b200.so in-tree (solargpu_b200/_lib/) for sm_100a.

    python -m solargpu_b200.build [--force]

CUDA sources are compiled with nvcc for ``-gencode arch=compute_100a,code=sm_100a``
(SASS only, with line info for profiling); host C++ with g++ and
``-ffp-contract=off`` so the host-side direction table is computed with the
same unfused float operations as the reference host code.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OUT = os.path.join(PKG, "_lib")
OBJ = os.path.join(OUT, "obj")
LIB = os.path.join(OUT, "libsolargpu_b200.so")

CU_SOURCES = ["trace.cu", "cone.cu", "barle.cu", "solar.cu", "reflect.cu", "group.cu", "tile.cu", "mma.cu", "voxel.cu",
              "pipeline.cu", "noalloc.cu", "surrogate.cu"]
CXX_SOURCES = ["sky.cpp", "cxx_api.cpp"]
HEADERS = ["sgb_internal.cuh", "solar_math.cuh", "sky.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    return shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def _cuda_include() -> str:
    return os.path.join(os.path.dirname(os.path.dirname(_nvcc())), "include")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str) -> str:
    path = os.path.join(CSRC, src)
    obj = os.path.join(OBJ, src + ".o")
    deps = [path] + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "solargpu_b200.h")]
    if not _stale(obj, deps):
        return obj
    inc = ["-I", CSRC, "-I", os.path.join(ROOT, "include")]
    if src.endswith(".cu"):
        cmd = [_nvcc(), "-std=c++17", "-O3", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
               *inc, "-c", path, "-o", obj]
    else:
        cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math", *inc,
               "-I", _cuda_include(), "-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every source and links the shared library; returns its path."""
    os.makedirs(OBJ, exist_ok=True)
    if force:
        for f in os.listdir(OBJ):
            os.remove(os.path.join(OBJ, f))
    srcs = CU_SOURCES + CXX_SOURCES
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(_compile, srcs))
    if force or _stale(LIB, objs):
        cmd = [_nvcc(), "-shared", *ARCH, "-cudart", "static", "-o", LIB, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
