"""Bounded device waits give up with an error status, never a hang.

The bulk-copy periodic steps (one cell per thread, and the staged FP16 step
with four) wait on shared-memory barriers for the rows they requested.  With OCTLB_TEST_BULK_STALL=1 one CTA skips requesting its first
row, so nothing ever completes that barrier: the wait runs out after
OCTLB_WAIT_MS, the CTA records the error word, drains the copies it did
request and returns, and the host reports OCTLB_ETIMEOUT.  The CUDA context
stays usable: a fresh lattice afterwards steps and matches the oracle.
(No fault is injected: the wait ends by its own limit.)
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bulk_step_wait_gives_up_with_etimeout(ob, orc, monkeypatch):
    from octlb_b200 import cases
    from oracle import oracle
    mesh, init, info = cases.tgv_periodic(64, u0=0.05, tau=0.55)
    monkeypatch.setenv("OCTLB_STEP_KERNEL", "bulk")
    monkeypatch.setenv("OCTLB_TEST_BULK_STALL", "1")
    monkeypatch.setenv("OCTLB_WAIT_MS", "50")
    lat = ob.GpuLattice(mesh, info["omega"], init_pops=init)
    lat.advance(2)
    with pytest.raises(ob.OctlbError) as e:
        lat.synchronize()
    assert e.value.code == ob.capi.OCTLB_ETIMEOUT, e.value
    assert "50 ms" in str(e.value)
    # every later read reports it too (the state is partly written)
    with pytest.raises(ob.OctlbError) as e:
        lat.audit()
    assert e.value.code == ob.capi.OCTLB_ETIMEOUT
    lat.close()

    # the same bulk step without the stall: correct, so the context survived
    monkeypatch.delenv("OCTLB_TEST_BULK_STALL")
    lat = ob.GpuLattice(mesh, info["omega"], init_pops=init)
    lat.advance(5)
    rho_g, u_g = lat.get_fields()
    lat.close()
    blk = oracle.Block(orc, 64)
    blk.set_core(init[0])
    blk.run_periodic(info["omega"], 5)
    rho_o, u_o = oracle.rho_u(blk.core())
    assert np.max(np.abs(u_g[0] - u_o)) <= 1e-5 * np.max(np.abs(u_o))


@pytest.mark.parametrize("order,prec", [("AB", "fp16"), ("AA", "fp16"), ("AA", "fp32")])
def test_staged_step_wait_gives_up_with_etimeout(ob, orc, monkeypatch, order, prec):
    """The same bounded wait in the staged periodic steps (the FP16 AB step
    with four cells per thread, and the AA order's pull step with its bulk
    stores in FP16 and FP32): the stalled CTA gives up, the host reports
    OCTLB_ETIMEOUT, and a fresh lattice afterwards steps correctly."""
    from octlb_b200 import cases
    from oracle import oracle
    mesh, init, info = cases.tgv_periodic(64, u0=0.05, tau=0.55)
    monkeypatch.setenv("OCTLB_TEST_BULK_STALL", "1")
    monkeypatch.setenv("OCTLB_WAIT_MS", "50")
    so = ob.ORDER_AA if order == "AA" else ob.ORDER_AB
    p = ob.FP16_SHIFTED if prec == "fp16" else ob.FP32
    lat = ob.GpuLattice(mesh, info["omega"], precision=p, init_pops=init, stream_order=so)
    lat.advance(2)
    with pytest.raises(ob.OctlbError) as e:
        lat.synchronize()
    assert e.value.code == ob.capi.OCTLB_ETIMEOUT, e.value
    lat.close()

    monkeypatch.delenv("OCTLB_TEST_BULK_STALL")
    lat = ob.GpuLattice(mesh, info["omega"], precision=p, init_pops=init, stream_order=so)
    lat.advance(5)
    rho_g, u_g = lat.get_fields()
    lat.close()
    blk = oracle.Block(orc, 64)
    blk.set_core(init[0])
    blk.run_periodic(info["omega"], 5)
    rho_o, u_o = oracle.rho_u(blk.core())
    assert np.max(np.abs(u_g[0] - u_o)) <= 2e-3 * np.max(np.abs(u_o))
