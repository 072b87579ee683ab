"""Bounded device waits give up with an error status, never a hang.

The bulk-copy periodic step waits on shared-memory barriers for the rows it
requested.  With OCTLB_TEST_BULK_STALL=1 one CTA skips requesting its first
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


def test_folded_coupler_wait_gives_up_with_etimeout(ob, monkeypatch):
    """A coupler launch folded into the next slot-map step's launch: with
    OCTLB_TEST_COUPLE_STALL=1 its CTAs never count themselves done, so each
    step CTA that reads a coupler target waits out OCTLB_WAIT_MS, records the
    error word and goes on; the host reports OCTLB_ETIMEOUT.  Afterwards a
    fresh lattice steps exactly as the stream-order schedule does (the
    context survived)."""
    from octlb_b200 import cases
    mesh, init, info = cases.cavity_forest(cells=16, n=8, lid=0.1, tau=0.6, band_cells=8)
    monkeypatch.setenv("OCTLB_TEST_COUPLE_STALL", "1")
    monkeypatch.setenv("OCTLB_WAIT_MS", "20")
    lat = ob.GpuLattice(mesh, info["omega"], init_pops=init)
    lat.advance(1)
    with pytest.raises(ob.OctlbError) as e:
        lat.synchronize()
    assert e.value.code == ob.capi.OCTLB_ETIMEOUT, e.value
    assert "coupler CTAs" in str(e.value) and "20 ms" in str(e.value)
    lat.close()

    monkeypatch.delenv("OCTLB_TEST_COUPLE_STALL")
    out = []
    for nofuse in ("0", "1"):
        monkeypatch.setenv("OCTLB_NO_FUSE", nofuse)
        lat = ob.GpuLattice(mesh, info["omega"], init_pops=init)
        lat.advance(3)
        out.append(lat.get_populations())
        lat.close()
    assert np.array_equal(out[0], out[1])
