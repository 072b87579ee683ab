"""The allocation-free audit entry point (octlb_gpu_audit_noalloc).

Some callers cannot call cudaMalloc: their device memory is owned by another
allocator, or they audit every step in a loop that cannot afford the device
synchronisation cudaMalloc / cudaFree imply.  This entry point keeps its
partial sums in a fixed device array inside the library instead.  Its output
must match the allocating octlb_gpu_audit on the same state, on two calls in a
row (the second call reuses the array the first one left behind).  This file
sorts last so that a run stopping at the first failure has run every other
test first; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12   # FP64 sums of the same values in a different order


def audit_noalloc(ob, lat):
    out = np.zeros(4)
    rc = ob.capi.lib().octlb_gpu_audit_noalloc(lat._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert rc == 0, ob.capi.lib().octlb_gpu_last_error(lat._h)
    return out


def close(a, b):
    return np.all(np.abs(a - b) <= TOL * max(1.0, np.max(np.abs(b))))


@pytest.mark.parametrize("case", ["tgv_fp32", "tgv_fp16", "amr_cavity"])
def test_audit_noalloc_matches_audit_twice(ob, case):
    from octlb_b200 import cases
    if case.startswith("tgv"):
        mesh, init, info = cases.tgv_periodic(64, u0=0.05, tau=0.55)
        prec = ob.FP32 if case == "tgv_fp32" else ob.FP16_SHIFTED
        lat = ob.GpuLattice(mesh, info["omega"], precision=prec, init_pops=init)
    else:
        mesh, init, info = cases.cavity_forest(cells=32, n=8, lid=0.1, tau=0.6, band_cells=8)
        lat = ob.GpuLattice(mesh, info["omega"], init_pops=init)
    lat.advance(7)
    for _ in range(2):
        ref = lat.audit()
        got = audit_noalloc(ob, lat)
        assert close(got, ref), (got, ref)
    lat.advance(3)
    assert close(audit_noalloc(ob, lat), lat.audit())
    lat.close()
