"""Rank contexts (octlb_gpu_create_part): the leaves shared over several
contexts, exchanging mirror cells before every level step and save rows
after it, here as rank contexts of one process on one GPU (the local
transport, one host thread per rank).  Their fields must equal the single
context's bit for bit (the exchange only copies values, every cell is
computed by the same kernel from the same inputs), their forces and audits
(sums over the ranks in another order) to 1e-12 relative; and the fields
must match the reference TimeLoop (oracle/_ref) to the FP32 tolerance.

A rank that never reaches an exchange ends the other ranks' calls with
OCTLB_ETIMEOUT after the transport's limit (host-side failure detection; no
device wait is involved)."""
import threading

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu


def run_ranks(ob, mesh, info, init, mode, drag, nranks, steps, prec, owner=None):
    owner = ob.partition(mesh, nranks) if owner is None else owner
    comm = ob.Comm.local(nranks)
    out = [None] * nranks
    errors = []

    def worker(r):
        try:
            lat = ob.GpuLattice(mesh, info["omega"], precision=prec, stream_mode=mode, drag=drag, init_pops=init,
                                part=(r, owner, comm))
            lat.advance(steps)
            lat.synchronize()
            rho, u = lat.get_fields()
            f = lat.force() if drag else None
            a = lat.audit()
            out[r] = (rho.copy(), u.copy(), f, a, lat.counters())
            lat.close()
        except Exception as e:  # reported by the test thread
            errors.append((r, e))

    th = [threading.Thread(target=worker, args=(r,)) for r in range(nranks)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    comm.close()
    assert not errors, errors
    rho = np.zeros_like(out[0][0])
    u = np.zeros_like(out[0][1])
    for r in range(nranks):
        m = owner == r
        rho[m] = out[r][0][m]
        u[m] = out[r][1][m]
    return rho, u, [o[2] for o in out], [o[3] for o in out], [o[4] for o in out], owner


CASES = {
    "cylinder": lambda c: (c.cylinder_forest(), 1, True),
    "amr_cavity": lambda c: (c.cavity_forest(cells=32, n=8, lid=0.1, tau=0.6, band_cells=8), 0, False),
}


@pytest.mark.parametrize("case", ["cylinder", "amr_cavity"])
@pytest.mark.parametrize("nranks", [2, 3, 4])
def test_rank_contexts_equal_one_context(ob, case, nranks):
    from octlb_b200 import cases
    (mesh, init, info), links, drag = CASES[case](cases)
    mode = ob.STREAM_LINKS if links else ob.STREAM_ROTATE
    steps = 12
    one = ob.GpuLattice(mesh, info["omega"], stream_mode=mode, drag=drag, init_pops=init)
    one.advance(steps)
    rho1, u1 = one.get_fields()
    f1 = one.force() if drag else None
    a1 = one.audit()
    c1 = one.counters()
    one.close()
    rho, u, fs, aus, cs, owner = run_ranks(ob, mesh, info, init, mode, drag, nranks, steps, ob.FP32)
    assert len(set(owner.tolist())) == nranks
    assert np.array_equal(rho, rho1) and np.array_equal(u, u1)
    for r in range(nranks):
        assert cs[r] == c1  # TimeLoop counters: every rank runs the whole recursion
        assert np.allclose(aus[r], a1, rtol=1e-12, atol=0)
        if drag:
            assert np.allclose(fs[r], f1, rtol=1e-12, atol=1e-15)
            assert np.array_equal(fs[r], fs[0])  # the same sum on every rank


def test_rank_contexts_fp16_and_reference(ob, ref):
    """Three rank contexts of the three-level cylinder in FP16-shifted
    storage equal one FP16 context bit for bit; in FP32 the two-level cavity
    split over two ranks matches the reference TimeLoop."""
    from octlb_b200 import cases
    mesh, init, info = cases.cylinder_forest()
    one = ob.GpuLattice(mesh, info["omega"], precision=ob.FP16_SHIFTED, stream_mode=ob.STREAM_LINKS, drag=True,
                        init_pops=init)
    one.advance(8)
    rho1, u1 = one.get_fields()
    one.close()
    rho, u, _, _, _, _ = run_ranks(ob, mesh, info, init, ob.STREAM_LINKS, True, 3, 8, ob.FP16_SHIFTED)
    assert np.array_equal(rho, rho1) and np.array_equal(u, u1)

    mesh, init, info = cases.cavity_forest(cells=16, n=8, lid=0.1, tau=0.6, band_cells=8)
    rho, u, _, _, _, _ = run_ranks(ob, mesh, info, init, ob.STREAM_ROTATE, False, 2, 10, ob.FP32)
    sim = oracle.Sim(ref, mesh, info["omega"], init)
    sim.advance(10)
    rho_r, u_r = oracle.rho_u(sim.core())
    assert np.max(np.abs(u - u_r)) <= 1e-5 * np.max(np.abs(u_r))
    assert np.max(np.abs(rho - rho_r)) <= 1e-5 * np.max(np.abs(rho_r))


def test_rank_that_never_arrives_times_out(ob, monkeypatch):
    """Rank 1 creates its context but never advances: rank 0's first exchange
    gives up after OCTLB_COMM_TIMEOUT_S (2 s) with OCTLB_ETIMEOUT."""
    from octlb_b200 import cases
    monkeypatch.setenv("OCTLB_COMM_TIMEOUT_S", "2")
    mesh, init, info = cases.cavity_forest(cells=16, n=8, lid=0.1, tau=0.6)
    owner = ob.partition(mesh, 2)
    comm = ob.Comm.local(2)
    lats = [ob.GpuLattice(mesh, info["omega"], init_pops=init, part=(r, owner, comm)) for r in range(2)]
    with pytest.raises(ob.OctlbError) as e:
        lats[0].advance(1)
    assert e.value.code == ob.capi.OCTLB_ETIMEOUT
    for lat in lats:
        lat.synchronize()
        lat.close()
    comm.close()


def run_slabs(ob, n, inits, omega, steps, prec=None):
    """Rank contexts of x slabs of a periodic box: inits[r] is slab r's
    initial populations (n^3 x 19); returns each slab's rho, u."""
    prec = ob.FP32 if prec is None else prec
    P = len(inits)
    comm = ob.Comm.local(P)
    mesh = ob.Mesh(n, [0], [0, 0, 0, 1, 1, 1], periodic=1)
    out, errors = [None] * P, []

    def worker(r):
        try:
            lat = ob.GpuLattice(mesh, omega, precision=prec, init_pops=inits[r], part=(r, np.zeros(1, np.int32), comm))
            lat.advance(steps)
            out[r] = lat.get_fields()
            lat.close()
        except Exception as e:
            errors.append((r, e))

    th = [threading.Thread(target=worker, args=(r,)) for r in range(P)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    comm.close()
    assert not errors, errors
    return out


@pytest.mark.parametrize("P", [2, 3])
def test_periodic_slabs_equal_one_box(ob, P):
    """P slabs holding the same Taylor-Green box form its periodic repetition:
    each slab's fields equal the single periodic box's bit for bit."""
    from octlb_b200 import cases
    n, steps = 32, 15
    mesh, init, info = cases.tgv_periodic(n, u0=0.05, tau=0.55)
    one = ob.GpuLattice(mesh, info["omega"], init_pops=init)
    one.advance(steps)
    rho1, u1 = one.get_fields()
    one.close()
    for rho, u in run_slabs(ob, n, [init] * P, info["omega"], steps):
        assert np.array_equal(rho, rho1) and np.array_equal(u, u1)


@pytest.mark.parametrize("rows", ["0", "2"])
def test_fp16_staged_step_on_slabs(ob, monkeypatch, rows):
    """The staged FP16 step on x slabs (its source rows at x - 1 and x + 1
    of the slab's first and last planes come from the ghost planes): two
    slabs holding the same box equal the single box stepped by the
    four-cell step with 8-byte global loads, bit for bit."""
    from octlb_b200 import cases
    n, steps = 32, 11
    mesh, init, info = cases.tgv_periodic(n, u0=0.05, tau=0.55)
    monkeypatch.setenv("OCTLB_FP16_ROWS", "off")
    one = ob.GpuLattice(mesh, info["omega"], precision=ob.FP16_SHIFTED, init_pops=init)
    one.advance(steps)
    rho1, u1 = one.get_fields()
    one.close()
    monkeypatch.setenv("OCTLB_FP16_ROWS", rows)
    for rho, u in run_slabs(ob, n, [init] * 2, info["omega"], steps, ob.FP16_SHIFTED):
        assert np.array_equal(rho, rho1) and np.array_equal(u, u1)


@pytest.mark.parametrize("prec,tol", [("fp32", 1e-5), ("fp16", 2e-3)])
def test_periodic_slabs_match_the_restated_box(ob, orc, prec, tol):
    """Two slabs of a 64 x 32 x 32 periodic box (one Taylor-Green period over
    the whole box in x, so the slabs differ) against the oracle's FP64 run of
    the whole box."""
    from octlb_b200 import cases
    n, steps, tau = 32, 40, 0.55
    rho0, u0 = cases.tgv_fields(2 * n, n, n, 0.05)
    f0 = ob.feq(rho0, u0)
    inits = [f0[:n][None], f0[n:][None]]
    slabs = run_slabs(ob, n, inits, 1.0 / tau, steps, ob.FP32 if prec == "fp32" else ob.FP16_SHIFTED)
    blk = oracle.Block(orc, 2 * n, n, n)
    blk.set_core(f0)
    blk.run_periodic(1.0 / tau, steps)
    rho_r, u_r = blk.fields()
    rho = np.concatenate([slabs[0][0][0], slabs[1][0][0]])
    u = np.concatenate([slabs[0][1][0], slabs[1][1][0]])
    assert np.max(np.abs(u - u_r)) <= tol * np.max(np.abs(u_r))
    assert np.max(np.abs(rho - rho_r)) <= tol * np.max(np.abs(rho_r))


@pytest.mark.parametrize("transport", ["local", "nccl"])
def test_single_slab_exchanging_with_itself(ob, transport):
    """One rank context of a periodic box, its ghost planes exchanged with
    itself -- through the local transport, and through NCCL (send / receive
    to the own rank, and the FP64 all-reduce of the audit): equal to the
    plain periodic box bit for bit.  The NCCL transport's only run on one
    GPU."""
    from octlb_b200 import cases
    n, steps = 32, 12
    mesh, init, info = cases.tgv_periodic(n, u0=0.05, tau=0.55)
    one = ob.GpuLattice(mesh, info["omega"], init_pops=init)
    one.advance(steps)
    rho1, u1 = one.get_fields()
    a1 = one.audit()
    one.close()
    comm = ob.Comm.local(1) if transport == "local" else ob.Comm.nccl(ob.Comm.nccl_unique_id(), 1, 0)
    lat = ob.GpuLattice(mesh, info["omega"], init_pops=init, part=(0, np.zeros(1, np.int32), comm))
    lat.advance(steps)
    lat.synchronize()
    rho, u = lat.get_fields()
    a = lat.audit()
    lat.close()
    comm.close()
    assert np.array_equal(rho, rho1) and np.array_equal(u, u1)
    assert np.array_equal(a, a1)
