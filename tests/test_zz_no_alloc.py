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


@pytest.mark.parametrize("case", ["tgv_fp32", "tgv_fp16", "tgv_fp32_aa", "amr_cavity"])
def test_audit_noalloc_matches_audit_twice(ob, case):
    from octlb_b200 import cases
    if case.startswith("tgv"):
        mesh, init, info = cases.tgv_periodic(64, u0=0.05, tau=0.55)
        prec = ob.FP16_SHIFTED if case == "tgv_fp16" else ob.FP32
        order = ob.ORDER_AA if case.endswith("_aa") else ob.ORDER_AB   # AA: 7 steps leave the reversed layout
        lat = ob.GpuLattice(mesh, info["omega"], precision=prec, init_pops=init, stream_order=order)
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


def test_audit_noalloc_rejects_levels_beyond_its_scratch(ob):
    """A level of more cells than the fixed array covers (33,554,432) is
    refused with OCTLB_EINVAL and a message that names the limit; nothing is
    launched.  A periodic 324^3 box (34,012,224 cells) in FP16 storage, at
    rest (no initial populations are uploaded)."""
    n = 324
    mesh = ob.Mesh(n, [0], [0, 0, 0, 1, 1, 1], periodic=1)
    lat = ob.GpuLattice(mesh, 1.0 / 0.55, precision=ob.FP16_SHIFTED)
    L = ob.capi.lib()
    out = np.zeros(4)
    rc = L.octlb_gpu_audit_noalloc(lat._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    msg = L.octlb_gpu_last_error(lat._h).decode()
    assert rc == ob.capi.OCTLB_EINVAL, (rc, msg)
    assert "33554432" in msg and str(n ** 3) in msg, msg
    # the allocating audit still covers it: the state at rest, mass = cells
    assert abs(lat.audit()[0] - n ** 3) <= 1e-9 * n ** 3
    lat.close()


def test_audit_noalloc_reports_a_bounded_wait_that_gave_up(ob, monkeypatch):
    """After a bounded device wait gave up (the test stall of the bulk-copy
    step: one CTA waits for a row it never requested, 50 ms limit), the
    allocation-free audit reports OCTLB_ETIMEOUT as octlb_gpu_audit does,
    instead of summing the partly written state."""
    from octlb_b200 import cases
    monkeypatch.setenv("OCTLB_STEP_KERNEL", "bulk")
    monkeypatch.setenv("OCTLB_TEST_BULK_STALL", "1")
    monkeypatch.setenv("OCTLB_WAIT_MS", "50")
    mesh, init, info = cases.tgv_periodic(64, u0=0.05, tau=0.55)
    lat = ob.GpuLattice(mesh, info["omega"], init_pops=init)
    lat.advance(1)
    L = ob.capi.lib()
    out = np.zeros(4)
    rc = L.octlb_gpu_audit_noalloc(lat._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert rc == ob.capi.OCTLB_ETIMEOUT, (rc, L.octlb_gpu_last_error(lat._h).decode())
    lat.close()
