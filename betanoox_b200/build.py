"""Builds the sm_100a shared library in-tree (betanoox_b200/_lib/libbeta_gpu.so).

nvcc cross-compiles for sm_100a without a GPU, so this runs on any machine
with the CUDA toolkit.  The library links the CUDA runtime statically and
exports only the C ABI declared in include/beta_gpu.h.
"""
from __future__ import annotations

import os
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libbeta_gpu.so")
SOURCES = ["beta_gpu.cu", "pattern.cpp", "exchange.cpp", "mesh_io.cpp", "surface_load.cpp", "element_groups.cpp"]

NVCC_FLAGS = [
    "-O3", "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-Xcompiler", "-fPIC,-pthread,-fvisibility=hidden,-Wall",
    "-shared", "-cudart", "static",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".cu", ".cuh", ".cpp", ".hpp", ".h"))]
    deps.append(os.path.join(HERE, "..", "include", "beta_gpu.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = [_nvcc(), *NVCC_FLAGS, "-o", LIB + ".tmp", *[os.path.join(SRC, s) for s in SOURCES]]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    started = time.time()
    subprocess.run(cmd, check=True)
    # the library carries the time its build started: a source edited while
    # nvcc ran (possibly after it had compiled that file) then reads as newer
    # and the next build() compiles everything again, instead of leaving
    # objects built from two versions of a shared header in one library
    os.utime(LIB + ".tmp", (started, started))
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
