"""Build libdimspers_b200.so in-tree with nvcc for sm_100a.

The library is plain C ABI (include/dimspers_b200.h); it links the CUDA
runtime statically so loading it needs no GPU.  Run as
``python -m dimspers_b200.build`` or through ``__graft_entry__.build()``.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libdimspers_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
         "-Xptxas", "-O3", "--expt-relaxed-constexpr"]


def sources():
    return [os.path.join(CSRC, "dimspers.cu"), os.path.join(CSRC, "mesh.cpp")]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    for f in os.listdir(CSRC):
        if os.path.getmtime(os.path.join(CSRC, f)) > t:
            return False
    hdr = os.path.join(HERE, "..", "include", "dimspers_b200.h")
    return os.path.getmtime(hdr) <= t


def build(force=False, verbose=False, extra=()):
    if not force and up_to_date():
        return LIB
    cmd = [NVCC, *ARCH, *FLAGS, *extra, "-shared", "-o", LIB, *sources()]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else [])
