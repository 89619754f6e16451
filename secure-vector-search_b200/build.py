"""Builds the sm_100a shared library of the BN backend in-tree.

    python secure-vector-search_b200/build.py

compiles every csrc/*.cu (and csrc/*.cpp) with nvcc into
bn_b200/libbn_b200.so next to the Python bindings, so the built library
travels with the repository snapshot.
"""
from __future__ import annotations

import glob
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
OUT = os.path.join(HERE, "bn_b200", "libbn_b200.so")
OBJ = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", f"-I{INCLUDE}", f"-I{CSRC}"]
HOST_CXX = ["-Xcompiler", "-O3", "-Xcompiler", "-march=x86-64-v3", "-Xcompiler", "-fopenmp",
            "-Xcompiler", "-ffp-contract=off"]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _digest(path: str, deps: list[str]) -> str:
    h = hashlib.sha256()
    for p in [path] + deps + [__file__]:
        with open(p, "rb") as f:
            h.update(f.read())
    h.update(" ".join(ARCH + COMMON + HOST_CXX).encode())
    return h.hexdigest()[:16]


def build(verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    headers = sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
                     + glob.glob(os.path.join(INCLUDE, "*.h")))
    objs = []
    for src in _sources():
        tag = _digest(src, headers)
        obj = os.path.join(OBJ, os.path.basename(src) + f".{tag}.o")
        if not os.path.exists(obj):
            cmd = [NVCC] + ARCH + COMMON + HOST_CXX + ["-c", src, "-o", obj]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
        objs.append(obj)
    link = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-Xcompiler", "-fopenmp", "-lcudart"]
    subprocess.run(link, check=True)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
