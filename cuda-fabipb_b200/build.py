"""Build libfabipb_b200.so in-tree (cuda-fabipb_b200/lib/) for sm_100a.

    python cuda-fabipb_b200/build.py [--force]

nvcc cross-compiles without a GPU, so this runs on any machine with CUDA 12.9.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libfabipb_b200.so")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_LIB = os.environ.get("CUDA_LIB", "/usr/local/cuda/lib64")


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    deps = glob.glob(os.path.join(CSRC, "*")) + glob.glob(os.path.join(HERE, "..", "include", "*.h"))
    if not force and not _newer(LIB, deps):
        return LIB
    out = None if verbose else subprocess.DEVNULL
    objs = []
    # host tree code: exact IEEE rounding, no contraction into FMA
    tree_o = os.path.join(BUILD, "tree.o")
    subprocess.run(["g++", "-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I/usr/local/cuda/include",
                    "-c", os.path.join(CSRC, "tree.cpp"), "-o", tree_o], check=True, stdout=out)
    objs.append(tree_o)
    abi_o = os.path.join(BUILD, "abi.o")
    if os.path.exists(os.path.join(CSRC, "abi.cpp")):
        subprocess.run(["g++", "-O3", "-std=c++17", "-fPIC", "-I/usr/local/cuda/include",
                        "-c", os.path.join(CSRC, "abi.cpp"), "-o", abi_o], check=True, stdout=out)
        objs.append(abi_o)
    main_o = os.path.join(BUILD, "fabipb_b200.o")
    subprocess.run([NVCC] + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                                    "-c", os.path.join(CSRC, "fabipb_b200.cu"), "-o", main_o],
                   check=True, stdout=out)
    objs.append(main_o)
    subprocess.run(["g++", "-shared", "-o", LIB] + objs +
                   ["-L" + CUDA_LIB, "-Wl,-rpath," + CUDA_LIB, "-lcudart", "-lcusolver", "-lpthread"],
                   check=True, stdout=out)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
