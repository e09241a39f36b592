"""Builds the UniformCUDA shared library in place (fluidsim_b200/libfluidcuda.so) for sm_100a."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBRARY = os.path.join(HERE, "libfluidcuda.so")
SOURCES = ["fc_engine.cu", "fc_server.cpp"]
# Every header beside the sources: a change to any of them rebuilds the library.
HEADERS = sorted(f for f in os.listdir(CSRC) if f.endswith((".cuh", ".h")))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
]


def _inputs():
    paths = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    paths.append(os.path.join(HERE, "..", "include", "fluidcuda.h"))
    return paths


def up_to_date() -> bool:
    if not os.path.exists(LIBRARY):
        return False
    built = os.path.getmtime(LIBRARY)
    return all(os.path.getmtime(p) <= built for p in _inputs())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIBRARY
    cmd = [NVCC] + FLAGS + [os.path.join(CSRC, s) for s in SOURCES] + ["-o", LIBRARY + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIBRARY + ".tmp", LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIBRARY)
