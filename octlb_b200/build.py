"""Builds the in-tree sm_100a shared library octlb_b200/liboctlb_b200.so.

The library holds the CUDA kernels, the host context behind the C ABI of
include/octlb_gpu.h and the host forest builder of include/octlb_forest.h.
It is built in place (not installed) so it travels with the source tree.
Each source compiles to its own object under _build/ (in parallel, rebuilt
when the source or a header is newer), then one link makes the library.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "liboctlb_b200.so")
OBJ = os.path.join(HERE, "..", "_build")
SOURCES = ["lbm_kernels.cu", "lbm_bulk.cu", "lbm_adjoint.cu", "lbm_exchange.cu", "lbm_fd.cu", "octlb_ctx.cu",
           "octlb_part.cu", "octlb_fd.cu", "forest.cpp", "vtk_writer.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo"] + ARCH + ["-Xcompiler", "-fPIC"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    inc = os.path.join(HERE, "..", "include")
    hs += [os.path.join(inc, f) for f in os.listdir(inc)]
    return hs


def _newest(paths):
    return max((os.path.getmtime(p) for p in paths if os.path.exists(p)), default=0.0)


def stale():
    if not os.path.exists(LIB):
        return True
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    return _newest(srcs + _headers()) > os.path.getmtime(LIB)


def _object(src, hdr_time, force):
    o = os.path.join(OBJ, os.path.basename(src) + ".o")
    if not force and os.path.exists(o) and os.path.getmtime(o) >= max(os.path.getmtime(src), hdr_time):
        return o, None
    cmd = [nvcc()] + NVCC_FLAGS + ["-c", "-o", o, src]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return o, (cmd, r)


def build(force=False, verbose=False):
    if not force and not stale():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    hdr_time = _newest(_headers())
    with ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _object(s, hdr_time, force), srcs))
    for o, res in results:
        if res is None:
            continue
        cmd, r = res
        if verbose:
            print(" ".join(cmd))
        if r.stdout or r.stderr:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode != 0:
            raise subprocess.CalledProcessError(r.returncode, cmd, r.stdout, r.stderr)
    cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + [o for o, _ in results]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
