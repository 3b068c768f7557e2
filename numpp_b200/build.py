"""Build recipe for libnumpp_b200.so (sm_100a kernels + C++20 host runtime + C ABI).

Compiles in-tree: objects under numpp_b200/_build/, the library at
numpp_b200/libnumpp_b200.so. Incremental on source/header timestamps.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libnumpp_b200.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INC = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def _cxx() -> str:
    return shutil.which("g++") or "g++"


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)


def build(verbose: bool = False, jobs: int = 8) -> str:
    os.makedirs(OUT, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.hpp")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "**", "*.h*"), recursive=True)
    cmds, objs = [], []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(OUT, os.path.basename(src) + ".o")
        objs.append(obj)
        if _newer(obj, [src] + headers):
            cmds.append([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                         *INC, "-c", src, "-o", obj])
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cpp"))):
        obj = os.path.join(OUT, os.path.basename(src) + ".o")
        objs.append(obj)
        if _newer(obj, [src] + headers):
            cmds.append([_cxx(), "-std=c++20", "-O2", "-fPIC", "-Wall", "-Wno-unused-function",
                         "-I" + os.path.join(CUDA, "include"), *INC, "-c", src, "-o", obj])
    procs = []
    for c in cmds:
        if verbose:
            print(" ".join(c), file=sys.stderr)
        procs.append(subprocess.Popen(c))
        if len(procs) >= jobs:
            if procs.pop(0).wait():
                raise RuntimeError("compile failed")
    for p in procs:
        if p.wait():
            raise RuntimeError("compile failed")
    if cmds or _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lpthread"], verbose)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
