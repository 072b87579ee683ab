"""The ctypes mirrors of the C ABI's structures (octlb_b200/capi.py) against
include/octlb_gpu.h: every field's offset and each structure's size, as a C
compiler lays them out, so the Python wrapper and a C caller pass the same
bytes (a field added to the header without its mirror fails here)."""
import ctypes
import os
import subprocess

import pytest

from octlb_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = {
    "octlb_params": capi.Params,
    "octlb_tables": capi.Tables,
    "octlb_adj_params": capi.AdjParams,
    "octlb_partition": capi.Partition,
    "octlb_fd_inlet": capi.FdInlet,
}


def c_layout(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "octlb_gpu.h"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return {(a, b): int(c) for a, b, c in (l.split() for l in out.splitlines())}


def test_ctypes_mirrors_match_the_header(tmp_path):
    lay = c_layout(tmp_path)
    for cname, py in STRUCTS.items():
        assert lay[(cname, "size")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert lay[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_stream_order_constants():
    with open(os.path.join(ROOT, "include", "octlb_gpu.h")) as f:
        text = f.read()
    assert "#define OCTLB_ORDER_AB 0" in text and "#define OCTLB_ORDER_AA 1" in text
    assert (capi.ORDER_AB, capi.ORDER_AA) == (0, 1)
