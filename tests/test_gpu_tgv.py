"""The throughput configuration's workload against FP64 runs of the
reference's algorithm, on the GPU through the C ABI:

* 64^3 Taylor-Green vortex (u0 = 0.05, tau = 0.55) for 1,000 steps against
  the reference's own BlockLattice<double> run
  (tests/golden/tgv64_reference.npz, tests/golden/make_tgv_reference.py):
  the kinetic-energy history every 10 steps and the final rho, u on a 16^3
  lattice of cells;
* the headline size itself, 256^3, for 10 steps against the oracle's C
  restatement of BlockLattice<double> (collide / fill_periodic_halo / stream,
  pinned to the reference build at 1e-13) run on the host threads: every
  cell's rho and u;
* octlb_gpu_set_equilibrium (the fields-to-state entry the end-to-end bench
  uses) equals octlb_gpu_set_populations of the same equilibrium.

Tolerances (max |gpu - ref| / max |ref| over the cells): FP32 rho, u 1e-5;
FP16-shifted 2e-3.  Kinetic energy (max over the history of |E_gpu - E_ref| /
E_ref): FP32 1e-5; FP16-shifted 2e-3.
"""
import os

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
TOL = {"fp32": 1e-5, "fp16": 2e-3}
KE_TOL = {"fp32": 1e-5, "fp16": 2e-3}


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def prec_of(ob, name):
    return ob.FP32 if name == "fp32" else ob.FP16_SHIFTED


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_tgv64_1000_steps_against_reference(ob, prec):
    from octlb_b200 import cases
    g = np.load(os.path.join(HERE, "golden", "tgv64_reference.npz"))
    n, every, steps = int(g["n"]), int(g["every"]), int(g["steps"])
    mesh, init, info = cases.tgv_periodic(n, u0=float(g["u0"]), tau=float(g["tau"]))
    lat = ob.GpuLattice(mesh, info["omega"], precision=prec_of(ob, prec), init_pops=init)
    ke, mass = [], []
    for k in range(steps // every + 1):
        if k:
            lat.advance(every)
        rho, u = lat.get_fields()
        ke.append(0.5 * float(np.sum(rho * np.sum(u * u, axis=-1))))
        mass.append(float(np.sum(rho)))
    lat.close()
    ke = np.array(ke)
    ke_err = float(np.max(np.abs(ke - g["ke"]) / g["ke"]))
    sl = (0, slice(2, None, 4), slice(2, None, 4), slice(2, None, 4))
    eu, er = rel(u[sl], g["sample_u"]), rel(rho[sl], g["sample_rho"])
    print(f"tgv64 {prec}: ke {ke_err:.2e} u {eu:.2e} rho {er:.2e} decay {ke[-1] / ke[0]:.6f} "
          f"(reference {g['ke'][-1] / g['ke'][0]:.6f})")
    assert ke_err <= KE_TOL[prec]
    assert eu <= TOL[prec] and er <= TOL[prec]
    # the periodic BGK conserves mass to rounding
    assert np.max(np.abs(np.array(mass) - g["mass"]) / g["mass"]) <= TOL[prec]
    # the field-wide sums of the reference run
    assert abs(float(np.sum(u * u)) - float(g["sum_u2"])) <= 2 * TOL[prec] * float(g["sum_u2"])


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_tgv256_headline_size_against_restatement(ob, orc, prec):
    from octlb_b200 import cases
    n, steps, tau = 256, 10, 0.55
    rho0, u0 = cases.tgv_fields(n, n, n, 0.05)
    mesh = ob.Mesh(n, [0], [0, 0, 0, 1, 1, 1], periodic=1)
    lat = ob.GpuLattice(mesh, 1.0 / tau, precision=prec_of(ob, prec))
    lat.set_equilibrium(rho0.reshape(-1), u0.reshape(-1, 3))
    lat.advance(steps)
    rho_g, u_g = lat.get_fields()
    lat.close()
    blk = oracle.Block(orc, n)
    blk.set_core(ob.feq(rho0, u0))
    blk.run_periodic_mt(1.0 / tau, steps)
    rho_r, u_r = blk.fields()
    del blk
    eu, er = rel(u_g[0], u_r), rel(rho_g[0], rho_r)
    print(f"tgv256 {prec}: u {eu:.2e} rho {er:.2e}")
    assert eu <= TOL[prec] and er <= TOL[prec]


@pytest.mark.parametrize("prec,n", [("fp32", 33), ("fp16", 33), ("fp32", 31)])
def test_odd_periodic_box_against_restatement(ob, orc, prec, n):
    """An odd block edge (no cell pairs: the one-cell-per-thread step on the
    periodic box) against the oracle's restatement of BlockLattice<double>,
    40 steps: every cell's rho and u."""
    from octlb_b200 import cases
    mesh, init, info = cases.tgv_periodic(n, u0=0.05, tau=0.55)
    lat = ob.GpuLattice(mesh, info["omega"], precision=prec_of(ob, prec), init_pops=init)
    lat.advance(40)
    rho_g, u_g = lat.get_fields()
    a = lat.audit()
    lat.close()
    blk = oracle.Block(orc, n)
    blk.set_core(init[0])
    blk.run_periodic(info["omega"], 40)
    rho_r, u_r = blk.fields()
    eu, er = rel(u_g[0], u_r), rel(rho_g[0], rho_r)
    print(f"periodic {n}^3 {prec}: u {eu:.2e} rho {er:.2e}")
    assert eu <= TOL[prec] and er <= TOL[prec]
    assert abs(a[0] - float(np.sum(rho_r))) <= TOL[prec] * n ** 3


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_set_equilibrium_equals_set_populations(ob, prec):
    from octlb_b200 import cases
    n = 32
    rho0, u0 = cases.tgv_fields(n, n, n, 0.05)
    mesh = ob.Mesh(n, [0], [0, 0, 0, 1, 1, 1], periodic=1)
    a = ob.GpuLattice(mesh, 1.0 / 0.55, precision=prec_of(ob, prec))
    b = ob.GpuLattice(mesh, 1.0 / 0.55, precision=prec_of(ob, prec))
    a.set_equilibrium(rho0.reshape(-1), u0.reshape(-1, 3))
    b.set_populations(ob.feq(rho0, u0))
    assert np.array_equal(a.get_populations(), b.get_populations())
    a.advance(3)
    b.advance(3)
    assert np.array_equal(a.get_populations(), b.get_populations())
    a.close()
    b.close()
    # a forest mesh (kinds, several blocks, two levels)
    mesh, init, info = cases.cavity_forest(cells=16, n=8, lid=0.1, tau=0.6, band_cells=8)
    rng = np.random.default_rng(7)
    cells = mesh.n_blocks * mesh.n ** 3
    rho = 1.0 + 0.01 * rng.standard_normal(cells)
    u = 0.03 * rng.standard_normal((cells, 3))
    a = ob.GpuLattice(mesh, info["omega"], precision=prec_of(ob, prec))
    b = ob.GpuLattice(mesh, info["omega"], precision=prec_of(ob, prec))
    a.set_equilibrium(rho, u)
    b.set_populations(ob.feq(rho, u))
    assert np.array_equal(a.get_populations(), b.get_populations())
    a.close()
    b.close()


@pytest.mark.parametrize("n", [32, 64, 128])
def test_fp16_four_cell_step_equals_paired_step(ob, monkeypatch, n):
    """The four-cells-per-thread FP16 periodic steps -- the one fed by bulk
    async copies through shared-memory stages in each of its launch shapes
    (OCTLB_FP16_ROWS: 64 to 256 threads, 2 or 3 stages, four or two cells per
    thread; whole z rows per stage, two copies per population at the y
    wrap), and
    the one with 8-byte global loads (OCTLB_FP16_ROWS=off) -- and the paired
    step (OCTLB_FP16_PAIR=1) give bitwise equal states."""
    from octlb_b200 import cases
    mesh, init, info = cases.tgv_periodic(n, u0=0.05, tau=0.55)
    out = []
    for pair, rows in (("1", "off"), ("0", "off"), ("0", "0"), ("0", "1"), ("0", "2"), ("0", "3"), ("0", "4"),
                       ("0", "5"), ("0", "6"), ("0", "7")):
        monkeypatch.setenv("OCTLB_FP16_PAIR", pair)
        monkeypatch.setenv("OCTLB_FP16_ROWS", rows)
        lat = ob.GpuLattice(mesh, info["omega"], precision=ob.FP16_SHIFTED, init_pops=init)
        lat.advance(7)
        out.append(lat.get_populations())
        lat.close()
    for k in range(1, len(out)):
        assert np.array_equal(out[0], out[k]), k


@pytest.mark.parametrize("prec,launch,n,pull", [("fp32", "graph", 64, None), ("fp16", "graph", 64, None),
                                                ("fp32", "direct", 64, None), ("fp16", "graph", 128, None),
                                                ("fp16", "direct", 128, "scalar"), ("fp16", "graph", 128, "quad"),
                                                ("fp16", "graph", 32, "rows1"), ("fp16", "direct", 64, "rows2"),
                                                ("fp32", "graph", 64, "scalar"), ("fp32", "graph", 32, "rows1"),
                                                ("fp32", "direct", 128, "rows2")])
def test_aa_order_equals_ab_order(ob, prec, launch, n, pull, monkeypatch):
    """The one-buffer AA stream order (a step that pulls from and writes back
    to the neighbours, then one on the cell's own slots, alternating) and the
    two-buffer AB order give bitwise equal populations, fields and audits
    after odd step counts (reversed layout) and even ones (natural layout),
    through captured graphs and direct launches, with each form of the pull
    step (by default staged through shared memory by bulk copies and stores,
    four FP16 or two FP32 cells per thread, in each launch shape,
    OCTLB_AA_ROWS; in FP16 four with shuffled aligned stores where a warp
    covers a 128-cell row, OCTLB_AA_PULL=quad, there with the unstaged local
    step too; one cell per thread, OCTLB_AA_PULL=scalar), and after
    set_populations while the AA buffer is in the reversed layout."""
    from octlb_b200 import cases
    if launch == "direct":
        monkeypatch.setenv("OCTLB_NO_GRAPH", "1")
    if pull and pull.startswith("rows"):
        monkeypatch.setenv("OCTLB_AA_ROWS", pull[4:])
    elif pull:
        monkeypatch.setenv("OCTLB_AA_PULL", pull)
        if pull == "quad":  # and the unstaged local step
            monkeypatch.setenv("OCTLB_FP16_ROWS", "off")
    mesh, init, info = cases.tgv_periodic(n, u0=0.05, tau=0.55)
    ab = ob.GpuLattice(mesh, info["omega"], precision=prec_of(ob, prec), init_pops=init)
    aa = ob.GpuLattice(mesh, info["omega"], precision=prec_of(ob, prec), init_pops=init, stream_order=ob.ORDER_AA)
    for k in (1, 6, 3):          # after 1, 7 and 10 steps
        ab.advance(k)
        aa.advance(k)
        assert np.array_equal(aa.get_populations(), ab.get_populations()), k
        ra, ua = aa.get_fields()
        rb, ub = ab.get_fields()
        assert np.array_equal(ra, rb) and np.array_equal(ua, ub), k
        assert np.array_equal(aa.audit(), ab.audit()), k
    aa.advance(1)
    ab.advance(1)                # 11 steps: reversed layout
    p = ab.get_populations()
    aa.set_populations(p)
    ab.set_populations(p)
    aa.advance(5)
    ab.advance(5)
    assert np.array_equal(aa.get_populations(), ab.get_populations())
    c_aa, s_aa = aa.counters()
    c_ab, s_ab = ab.counters()
    assert c_aa == c_ab and s_aa == s_ab
    ab.close()
    aa.close()


def test_aa_order_holds_one_buffer(ob):
    """AA keeps one population buffer: creating the 128^3 FP32 box takes about
    half the device memory of the AB order (2 x 159 MB)."""
    import torch
    from octlb_b200 import cases
    mesh, init, info = cases.tgv_periodic(128, u0=0.05, tau=0.55)
    used = {}
    for order in (ob.ORDER_AB, ob.ORDER_AA):
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        lat = ob.GpuLattice(mesh, info["omega"], stream_order=order)
        torch.cuda.synchronize()
        used[order] = free0 - torch.cuda.mem_get_info()[0]
        lat.close()
    one = 128 ** 3 * 19 * 4
    assert used[ob.ORDER_AB] >= 2 * one
    assert used[ob.ORDER_AA] < used[ob.ORDER_AB] - 0.9 * one


def test_aa_order_refusals(ob):
    """AA runs the uniform periodic box only, without body force or
    ConstRhoBGK (OCTLB_EINVAL)."""
    from octlb_b200 import cases
    mesh, init, info = cases.cavity_forest(cells=16, n=8, lid=0.1, tau=0.6)
    with pytest.raises(ob.OctlbError):
        ob.GpuLattice(mesh, info["omega"], stream_order=ob.ORDER_AA)
    mesh, init, info = cases.tgv_periodic(32, u0=0.05, tau=0.55)
    with pytest.raises(ob.OctlbError):
        ob.GpuLattice(mesh, info["omega"], stream_order=7)
    lat = ob.GpuLattice(mesh, info["omega"], init_pops=init, stream_order=ob.ORDER_AA)
    with pytest.raises(ob.OctlbError):
        lat.set_body_force(np.zeros((1, 32 ** 3, 3)))
    with pytest.raises(ob.OctlbError):
        lat.set_const_rho(True)
    lat.advance(3)
    assert np.all(np.isfinite(lat.get_populations()))
    lat.close()
