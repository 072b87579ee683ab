"""Builds the in-tree sm_100a shared library octlb_b200/liboctlb_b200.so.

The library holds the CUDA kernels, the host context behind the C ABI of
include/octlb_gpu.h and the host forest builder of include/octlb_forest.h.
It is built in place (not installed) so it travels with the source tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "liboctlb_b200.so")
SOURCES = ["lbm_kernels.cu", "lbm_bulk.cu", "lbm_adjoint.cu", "octlb_ctx.cu", "forest.cpp", "vtk_writer.cpp"]
NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "octlb_gpu.h"))
    deps.append(os.path.join(HERE, "..", "include", "octlb_forest.h"))
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    if not force and not stale():
        return LIB
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    cmd = [nvcc()] + NVCC_FLAGS + ["-o", LIB] + srcs
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
