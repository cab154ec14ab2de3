"""Build the backend's shared library (libg2o_b200.so, in-tree) with nvcc for
sm_100a. The C-ABI of include/g2o_cuda.h is its only interface."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libg2o_b200.so")
CLI = os.path.join(HERE, "g2o_cuda_cli")
CLI_SOURCE = "g2o_cuda_cli.cpp"
SOURCES = ["g2oc_api.cu", "noalloc.cu", "structure.cpp", "g2o_io.cpp"]
HEADERS = sorted(f for f in os.listdir(CSRC) if f.endswith((".h", ".cuh")))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", "-Xcompiler", "-fopenmp",
         "--expt-relaxed-constexpr", "-ccbin", "/usr/bin/g++"]


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths)


def up_to_date() -> bool:
    if not os.path.exists(LIB) or not os.path.exists(CLI):
        return False
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS + [CLI_SOURCE]]
    deps += [os.path.join(HERE, "..", "include", h) for h in ("g2o_cuda.h", "g2o_io.h")]
    deps.append(__file__)
    return min(os.path.getmtime(LIB), os.path.getmtime(CLI)) >= _newest(deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    objs = []
    for src in SOURCES:
        obj = os.path.join(CSRC, os.path.splitext(src)[0] + ".o")
        cmd = [NVCC] + ARCH + FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [NVCC] + ARCH + ["-shared", "-ccbin", "/usr/bin/g++", "-o", LIB] + objs + ["-lcudart", "-lgomp"]
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    # the command-line optimizer, linked against the library next to it
    cmd = ["/usr/bin/g++", "-std=c++17", "-O2", "-o", CLI, os.path.join(CSRC, CLI_SOURCE), "-L" + HERE,
           "-lg2o_b200", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
