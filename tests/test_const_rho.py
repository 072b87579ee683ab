"""ConstRhoBGK (the reference TimeLoop's use_const_rho_bgk): the collide of
block_lattice.cpp:441-455 / block_lattice.h:134-151 with the average density
of the previous collide's statistics (time_loop.h:201-222).

CPU: the reference build's statistics against their definition.  GPU (through
the C ABI): fields and average_rho against the reference TimeLoop run with
use_const_rho_bgk, on single-level meshes under both stream rules and on two-
and three-level meshes (statistics of the finest level, every level colliding
at the average); FP32 tolerance 1e-5, FP16-shifted 2e-3 (max-abs over
max-abs), average_rho within 1e-6 (FP32; the GPU sums FP32 densities in
FP64)."""
import numpy as np
import pytest

from oracle import oracle

TOL32 = 1e-5
TOL16 = 2e-3


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def rest_state(mesh, rho):
    """Shifted equilibrium at rest with density rho [n_blocks][n][n][n]."""
    from octlb_b200 import C
    Cf = C.astype(np.float64)
    w = np.where(np.abs(Cf).sum(1) == 0, 1 / 3, np.where(np.abs(Cf).sum(1) == 1, 1 / 18, 1 / 36))
    return np.ascontiguousarray(w * rho[..., None] - w)


def brick_cavity(lid=0.1, tau=0.6, n=8):
    """Cavity of 2 x 2 x 2 level-0 blocks (one collide per advance_one), walls
    on every tree boundary, +y wall moving with (lid, 0, 0)."""
    from octlb_b200 import Forest, Mesh, TB_WALL, cases
    f = Forest((2, 2, 2), (0, 0, 0), (0, 0, 0, 1, 1, 1)).balance().build()

    def spec(b, d):
        return [TB_WALL, lid if d == 3 else 0.0, 0, 0, -1, 0, 0, 0]

    mesh = Mesh.from_forest(f, n, tree_boundary_spec=cases._tb_spec(f, spec))
    return mesh, {"omega": 1.0 / tau}


def perturbed_density(mesh, mean, seed):
    n = mesh.n
    rng = np.random.default_rng(seed)
    return mean + 0.01 * rng.standard_normal((mesh.n_blocks, n, n, n))


def test_reference_const_rho_statistics(ref):
    """One collide from a state at rest: average_rho becomes the mean density
    of the kBulk cells (statistic rho + (1 - 1)); the next collide adds
    1 - average_rho to every kBulk cell's density."""
    mesh, info = brick_cavity()
    rho0 = perturbed_density(mesh, 1.02, 3)
    init = rest_state(mesh, rho0)
    sim = oracle.Sim(ref, mesh, info["omega"], init)
    sim.set_const_rho(True)
    assert sim.average_rho() == 1.0
    sim.advance(1)
    bulk = mesh.kinds == 0
    a1 = sim.average_rho()
    assert abs(a1 - rho0[bulk].mean()) <= 1e-12
    rho_before, _ = oracle.rho_u(sim.core())
    sim.advance(1)
    # the second collide's statistic: its pre-collision density (the
    # post-stream state after call 1) plus 1 - a1
    assert abs(sim.average_rho() - (rho_before[bulk].mean() + 1.0 - a1)) <= 1e-12
    bgk = oracle.Sim(ref, mesh, info["omega"], init)
    bgk.advance(2)
    assert bgk.average_rho() == 1.0
    # the collide took the density toward 1
    rho_cr, _ = oracle.rho_u(sim.core())
    rho_bgk, _ = oracle.rho_u(bgk.core())
    assert abs(rho_cr[bulk].mean() - 1.0) < 0.2 * abs(rho_bgk[bulk].mean() - 1.0)


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol,kernel", [("fp32", TOL32, "map"), ("fp16", TOL16, "map"), ("fp32", TOL32, "plain")])
def test_const_rho_cavity_matches_reference(ob, ref, prec, tol, kernel, monkeypatch):
    """Moving-lid cavity, torus-rotate stream rule with wall fills, from a
    perturbed rest state at mean density 1.02: average_rho after every call
    and the fields after 1 and 12 calls against the reference TimeLoop (the
    slot-map step and the plain step)."""
    if kernel == "plain":
        monkeypatch.setenv("OCTLB_STEP_KERNEL", "plain")
    mesh, info = brick_cavity()
    init = rest_state(mesh, perturbed_density(mesh, 1.02, 5))
    lat = ob.GpuLattice(mesh, info["omega"], precision=ob.FP32 if prec == "fp32" else ob.FP16_SHIFTED,
                        init_pops=init)
    lat.set_const_rho(True)
    sim = oracle.Sim(ref, mesh, info["omega"], init)
    sim.set_const_rho(True)
    bgk = oracle.Sim(ref, mesh, info["omega"], init)
    atol = 1e-6 if prec == "fp32" else 2e-4
    for call in range(12):
        lat.advance(1)
        sim.advance(1)
        bgk.advance(1)
        assert abs(lat.average_rho() - sim.average_rho()) <= atol, call
        if call in (0, 11):
            rho_g, u_g = lat.get_fields()
            rho_r, u_r = oracle.rho_u(sim.core())
            assert rel(rho_g, rho_r) <= tol, call
            assert rel(u_g, u_r) <= tol, call
    # ConstRhoBGK and BGK part well beyond the tolerance
    rho_b, u_b = oracle.rho_u(bgk.core())
    assert rel(rho_b, rho_r) > 100 * TOL32
    c, s = lat.counters()
    cr, sr, _ = sim.counters()
    assert c == cr and s == sr
    lat.close()


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["map", "plain"])
def test_const_rho_cylinder_links_matches_reference(ob, ref, kernel, monkeypatch):
    """Single-level channel with a Bouzidi cylinder (links stream rule, near-wall
    cells on their own warps, parabolic moving-wall inlet, outflow copy),
    from a perturbed rest state at mean density 1.01."""
    if kernel == "plain":
        monkeypatch.setenv("OCTLB_STEP_KERNEL", "plain")
    from octlb_b200 import cases
    mesh, init0, info = cases.cylinder_forest(length=64, height=32, n=8, diameter=8.0, center=(16.0, 16.0),
                                              levels=1)
    assert len(set(mesh.levels.tolist())) == 1
    rho0 = perturbed_density(mesh, 1.01, 9)
    init = rest_state(mesh, rho0)
    init[mesh.kinds == ob.SOLID] = 0.0
    lat = ob.GpuLattice(mesh, info["omega"], stream_mode=ob.STREAM_LINKS, init_pops=init)
    lat.set_const_rho(True)
    sim = oracle.Sim(ref, mesh, info["omega"], init, link_mode=True)
    sim.set_const_rho(True)
    for call in range(3):
        lat.advance(1)
        sim.advance(1)
        assert abs(lat.average_rho() - sim.average_rho()) <= 1e-6, call
    rho_g, u_g = lat.get_fields()
    rho_r, u_r = oracle.rho_u(sim.core())
    fl = mesh.kinds != ob.SOLID
    assert rel(rho_g[fl], rho_r[fl]) <= TOL32
    assert rel(u_g[fl], u_r[fl]) <= TOL32
    lat.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol,kernel", [("fp32", TOL32, "map"), ("fp16", TOL16, "map"), ("fp32", TOL32, "plain")])
def test_const_rho_amr_cavity_matches_reference(ob, ref, prec, tol, kernel, monkeypatch):
    """Two-level moving-lid cavity (16^3 base, refined band under the lid)
    from a perturbed rest state at mean density 1.02: the statistics are the
    finest level's collides (prolongation targets included, with the
    densities the prolongation wrote), the coarse level collides at the same
    average (time_loop.h:201-222); average_rho after every call and the fields
    of both levels after 1 and 12 calls against the reference TimeLoop."""
    if kernel == "plain":
        monkeypatch.setenv("OCTLB_STEP_KERNEL", "plain")
    from octlb_b200 import cases
    mesh, _, info = cases.cavity_forest(cells=16, n=8, lid=0.1, tau=0.6, band_cells=8)
    assert len(set(mesh.levels.tolist())) == 2
    init = rest_state(mesh, perturbed_density(mesh, 1.02, 17))
    lat = ob.GpuLattice(mesh, info["omega"], precision=ob.FP32 if prec == "fp32" else ob.FP16_SHIFTED,
                        init_pops=init)
    lat.set_const_rho(True)
    sim = oracle.Sim(ref, mesh, info["omega"], init)
    sim.set_const_rho(True)
    bgk = oracle.Sim(ref, mesh, info["omega"], init)
    atol = 1e-6 if prec == "fp32" else 2e-4
    for call in range(12):
        lat.advance(1)
        sim.advance(1)
        bgk.advance(1)
        assert abs(lat.average_rho() - sim.average_rho()) <= atol, call
        if call in (0, 11):
            rho_g, u_g = lat.get_fields()
            rho_r, u_r = oracle.rho_u(sim.core())
            assert rel(rho_g, rho_r) <= tol, call
            assert rel(u_g, u_r) <= tol, call
    rho_b, _ = oracle.rho_u(bgk.core())
    assert rel(rho_b, rho_r) > 100 * TOL32
    c, s = lat.counters()
    cr, sr, _ = sim.counters()
    assert c == cr and s == sr
    lat.close()


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["map", "plain"])
def test_const_rho_three_level_cylinder_matches_reference(ob, ref, kernel, monkeypatch):
    """Three-level channel with a Bouzidi cylinder (links stream rule, near-wall
    cells, parabolic inlet, outflow copy) from a perturbed rest state at mean
    density 1.01: two levels above the finest stream, couple and then collide
    at the average of the finest level's statistics."""
    if kernel == "plain":
        monkeypatch.setenv("OCTLB_STEP_KERNEL", "plain")
    from octlb_b200 import cases
    mesh, _, info = cases.cylinder_forest(length=128, height=32, n=8, diameter=8.0, center=(16.0, 16.0), levels=3,
                                          refine_dist=8.0)
    assert len(set(mesh.levels.tolist())) == 3
    init = rest_state(mesh, perturbed_density(mesh, 1.01, 23))
    init[mesh.kinds == ob.SOLID] = 0.0
    lat = ob.GpuLattice(mesh, info["omega"], stream_mode=ob.STREAM_LINKS, init_pops=init)
    lat.set_const_rho(True)
    sim = oracle.Sim(ref, mesh, info["omega"], init, link_mode=True)
    sim.set_const_rho(True)
    for call in range(4):
        lat.advance(1)
        sim.advance(1)
        assert abs(lat.average_rho() - sim.average_rho()) <= 1e-6, call
    rho_g, u_g = lat.get_fields()
    rho_r, u_r = oracle.rho_u(sim.core())
    fl = mesh.kinds != ob.SOLID
    assert rel(rho_g[fl], rho_r[fl]) <= TOL32
    assert rel(u_g[fl], u_r[fl]) <= TOL32
    lat.close()


@pytest.mark.gpu
def test_const_rho_argument_checks(ob):
    from octlb_b200 import cases
    mesh, init, info = cases.cavity_forest(cells=16, n=8, lid=0.1, tau=0.6, band_cells=8)
    two = ob.GpuLattice(mesh, info["omega"], init_pops=init)
    assert two.average_rho() == 1.0
    two.set_const_rho(True)                  # two levels: the finest level's statistics
    two.advance(1)
    assert two.average_rho() != 1.0
    with pytest.raises(ob.OctlbError):
        two.adjoint(4, 2)                    # the adjoint differentiates BGK
    two.close()
    mesh, info = brick_cavity()
    lat = ob.GpuLattice(mesh, info["omega"])
    lat.set_const_rho(True)
    lat.set_const_rho(False)                 # still before the first advance
    lat.set_const_rho(True)
    lat.advance(1)
    with pytest.raises(ob.OctlbError):
        lat.set_const_rho(False)             # after the first advance
    lat.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol,atol", [("fp32", TOL32, 1e-9), ("fp16", TOL16, 1e-6)])
def test_const_rho_long_run_matches_reference(ob, ref, prec, tol, atol):
    """1,000 ConstRhoBGK steps of the moving-lid cavity from a perturbed rest
    state at mean density 1.02: the density held at 1 by the average-density
    feedback and the flow the lid drives, against the reference TimeLoop
    (max-abs over max-abs: 1e-5 FP32, 2e-3 FP16-shifted; measured 6.6e-7 and
    5.6e-4 on u), and average_rho (within 1e-9 FP32, 1e-6 FP16)."""
    mesh, info = brick_cavity()
    init = rest_state(mesh, perturbed_density(mesh, 1.02, 21))
    lat = ob.GpuLattice(mesh, info["omega"], precision=ob.FP32 if prec == "fp32" else ob.FP16_SHIFTED,
                        init_pops=init)
    lat.set_const_rho(True)
    sim = oracle.Sim(ref, mesh, info["omega"], init)
    sim.set_const_rho(True)
    lat.advance(1000)
    sim.advance(1000)
    rho_g, u_g = lat.get_fields()
    rho_r, u_r = oracle.rho_u(sim.core())
    assert rel(rho_g, rho_r) <= tol
    assert rel(u_g, u_r) <= tol
    assert abs(lat.average_rho() - sim.average_rho()) <= atol
    assert abs(rho_r[mesh.kinds == 0].mean() - 1.0) < 1e-3   # held at unit density
    assert np.abs(u_r).max() > 0.01                           # the lid drives the flow
    lat.close()
