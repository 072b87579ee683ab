"""Finite-difference domain boundary conditions on the GPU
(octlb_gpu_set_fd_boundary) against the reference's own
ConcreteDomainBoundaryHandler in the reference TimeLoop (oracle/_ref,
oracle.Sim.set_fd_boundary): the fields after N steps, FP32 <= 1e-5 relative
(max |gpu - ref| / max |ref| over all cells), FP16-shifted <= 2e-3.

* cavity3d's boundary: InterpolatedVelocity on every face, the y+ face's
  wall velocity on the interior lid cells (one 16^3 block, and one 31^3
  block as the example runs it);
* a channel: a uniform inlet on x- ramped over 20 steps, a pressure outlet
  on x+ (target density 1), velocity walls elsewhere;
* eight 8^3 blocks (the roles of a block's rim cells come from its own
  extents, as in the reference), with the lid or with a pressure outlet
  spanning four blocks;
* two-level meshes (the pass after every level's step);
* a rest state stays exactly at rest."""
import os
import sys

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
S = oracle.Sim


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def run_pair(ob, ref, mesh, init, omega, types, u, rho_t, steps, prec, inlet=None, ramp=0.0):
    stamped = ob.stamp_fd_kinds(mesh, types)
    lat = ob.GpuLattice(stamped, omega, precision=prec, init_pops=init)
    lat.set_fd_boundary(types, u, rho_t, inlet, ramp)
    lat.advance(steps)
    rho_g, u_g = lat.get_fields()
    lat.close()
    sim = S(ref, mesh, omega, init)
    sim.set_fd_boundary(types, u, rho_target=rho_t, inlet_u=inlet, ramp_end_t=ramp)
    sim.advance(steps)
    rho_r, u_r = oracle.rho_u(sim.core())
    return rho_g, u_g, rho_r, u_r


@pytest.mark.parametrize("prec,tol,n", [("fp32", 1e-5, 16), ("fp16", 2e-3, 16), ("fp32", 1e-5, 31),
                                        ("fp16", 2e-3, 31)])
def test_cavity3d_boundary(ob, ref, prec, tol, n):
    """cavity3d's walls and lid on one block: 16^3, and the example's own
    31^3 lattice (an odd block edge: the one-cell-per-thread step)."""
    from octlb_b200 import cases
    mesh, init, info = cases.cavity_forest(cells=n, n=n, lid=0.0, tau=0.6)
    u = np.zeros((6, 3))
    u[3, 0] = 0.05
    rho_g, u_g, rho_r, u_r = run_pair(ob, ref, mesh, init, info["omega"], [S.INTERPOLATED_VELOCITY] * 6, u,
                                      np.ones(6), 60, ob.FP32 if prec == "fp32" else ob.FP16_SHIFTED)
    print(f"fd cavity {prec}: u {rel(u_g, u_r):.2e} rho {rel(rho_g, rho_r):.2e}")
    assert np.abs(u_r).max() > 0.01
    assert rel(u_g, u_r) <= tol and rel(rho_g, rho_r) <= tol


def test_inlet_and_pressure_outlet(ob, ref):
    from octlb_b200 import cases
    mesh, init, info = cases.cavity_forest(cells=16, n=16, lid=0.0, tau=0.6)
    types = [S.INTERPOLATED_VELOCITY, S.INTERPOLATED_PRESSURE] + [S.INTERPOLATED_VELOCITY] * 4
    inlet = np.zeros((6, 3))
    inlet[0, 0] = 0.02
    rho_g, u_g, rho_r, u_r = run_pair(ob, ref, mesh, init, info["omega"], types, np.zeros((6, 3)), np.ones(6), 40,
                                      ob.FP32, inlet, 20.0)
    print(f"fd channel: u {rel(u_g, u_r):.2e} rho {rel(rho_g, rho_r):.2e}")
    assert np.abs(u_r).max() > 0.005
    assert rel(u_g, u_r) <= 1e-5 and rel(rho_g, rho_r) <= 1e-5


@pytest.mark.parametrize("inlet", [None, "uniform", "poiseuille", "channel"])
def test_eight_blocks(ob, ref, inlet):
    """Eight 8^3 blocks: the lid, or an inlet on x- against a pressure outlet
    on x+ that spans four blocks (its block-rim cells read u = 0 and
    density 1, as the reference's view does off a flat face).  The inlet is
    uniform, or one of the reference's duct fields: parabolas over each
    block's in-plane indices (PoiseuilleInletProfile) or over a physical
    patch of the face (ChannelPoiseuilleInletProfile, cylinder3d's inlet)."""
    sys.path.insert(0, HERE)
    from test_const_rho import brick_cavity
    mesh, info = brick_cavity(lid=0.0, n=8)
    init = np.zeros((mesh.n_blocks, 8, 8, 8, 19))
    types = [S.INTERPOLATED_VELOCITY] * 6
    u = np.zeros((6, 3))
    rho_t = np.ones(6)
    if inlet is None:
        u[3, 0] = 0.05
        rho_g, u_g, rho_r, u_r = run_pair(ob, ref, mesh, init, info["omega"], types, u, rho_t, 30, ob.FP32)
    else:
        types[1] = S.INTERPOLATED_PRESSURE
        rho_t[1] = 1.002
        if inlet == "uniform":
            spec = ob.fd_inlet(ob.INLET_UNIFORM, (0.02, 0.0, 0.0), ramp_end_t=10.0)
        else:
            kind = ob.INLET_POISEUILLE if inlet == "poiseuille" else ob.INLET_CHANNEL_POISEUILLE
            spec = ob.fd_inlet(kind, (1.0, 0.0, 0.0), 0.04, (8, 8), (0.1, 0.9, 0.2, 0.8), 10.0)
        inlets = [spec] + [None] * 5
        lat = ob.GpuLattice(ob.stamp_fd_kinds(mesh, types), info["omega"], init_pops=init)
        lat.set_fd_boundary(types, u, rho_t, inlets=inlets)
        lat.advance(30)
        rho_g, u_g = lat.get_fields()
        lat.close()
        sim = S(ref, mesh, info["omega"], init)
        sim.set_fd_boundary(types, u, rho_target=rho_t, inlets=inlets)
        sim.advance(30)
        rho_r, u_r = oracle.rho_u(sim.core())
    print(f"fd 8 blocks (inlet {inlet}): u {rel(u_g, u_r):.2e} rho {rel(rho_g, rho_r):.2e}")
    assert np.abs(u_r).max() > 0.004
    assert rel(u_g, u_r) <= 1e-5 and rel(rho_g, rho_r) <= 1e-5


def test_rest_state_is_a_fixed_point(ob):
    from octlb_b200 import cases
    mesh, init, info = cases.cavity_forest(cells=16, n=16, lid=0.0, tau=0.6)
    types = [S.INTERPOLATED_VELOCITY] * 6
    lat = ob.GpuLattice(ob.stamp_fd_kinds(mesh, types), info["omega"], init_pops=init)
    lat.set_fd_boundary(types)
    lat.advance(10)
    assert np.abs(lat.get_populations()).max() == 0.0
    lat.close()


@pytest.mark.parametrize("blocks", [1, 8, "31"])
def test_const_rho_with_fd_walls(ob, ref, blocks):
    """cavity3d's configuration: ConstRhoBGK in the bulk with the FD walls
    and lid, the velocity cells' collide densities in the average's
    statistics (kFluidAndBoundary): fields and average_rho after every few
    steps against the reference TimeLoop built with use_const_rho_bgk around
    the reference's handler.  Eight blocks also exercise the stencils'
    reads of kBulk densities, which carry the collide's 1 - average_rho;
    "31" is cavity3d's own lattice, one 31^3 block (RESOLUTION = 30, an odd
    block edge)."""
    from octlb_b200 import cases
    if blocks in (1, "31"):
        c = 16 if blocks == 1 else 31
        mesh, init, info = cases.cavity_forest(cells=c, n=c, lid=0.0, tau=0.6)
        omega = info["omega"]
    else:
        sys.path.insert(0, HERE)
        from test_const_rho import brick_cavity
        mesh, info = brick_cavity(lid=0.0, n=8)
        init = np.zeros((mesh.n_blocks, 8, 8, 8, 19))
        omega = info["omega"]
    types = [S.INTERPOLATED_VELOCITY] * 6
    u = np.zeros((6, 3))
    u[3, 0] = 0.05
    lat = ob.GpuLattice(ob.stamp_fd_kinds(mesh, types), omega, init_pops=init)
    lat.set_const_rho(True)
    lat.set_fd_boundary(types, u)
    sim = S(ref, mesh, omega, init)
    sim.set_fd_boundary(types, u, const_rho=True)
    for _ in range(4):
        lat.advance(10)
        sim.advance(10)
        rho_g, u_g = lat.get_fields()
        rho_r, u_r = oracle.rho_u(sim.core())
        eu, er = rel(u_g, u_r), rel(rho_g, rho_r)
        da = abs(lat.average_rho() - sim.average_rho())
        print(f"fd const rho ({blocks} blocks): u {eu:.2e} rho {er:.2e} average_rho {da:.2e}")
        assert eu <= 1e-5 and er <= 1e-5 and da <= 1e-6
    lat.close()


def test_no_slip_walls_and_moving_lid_types(ob, ref):
    """The handler's other domain types: no-slip walls (kBounceBack, the
    dispatcher's full-way swap at collide) on five faces and an
    InterpolatedVelocity lid; then the lid as a moving-lid face (no
    collide-time action) over outflow side faces."""
    from octlb_b200 import cases
    mesh, init, info = cases.cavity_forest(cells=16, n=16, lid=0.0, tau=0.6)
    u = np.zeros((6, 3))
    u[3, 0] = 0.05
    for types in ([S.NO_SLIP] * 3 + [S.INTERPOLATED_VELOCITY] + [S.NO_SLIP] * 2,
                  [S.OUTFLOW, S.OUTFLOW, S.NO_SLIP, S.MOVING_LID, S.INTERPOLATED_VELOCITY,
                   S.INTERPOLATED_VELOCITY]):
        rho_g, u_g, rho_r, u_r = run_pair(ob, ref, mesh, init, info["omega"], types, u, np.ones(6), 30, ob.FP32)
        print(f"fd types {types}: u {rel(u_g, u_r):.2e} rho {rel(rho_g, rho_r):.2e}")
        assert rel(u_g, u_r) <= 1e-5 and rel(rho_g, rho_r) <= 1e-5


def interior_refined_cavity(ob, nested=False):
    """32^3 cavity in 8^3 blocks (forest level 2) with its central 2 x 2 x 2
    blocks refined one level (nested: and the centre of those once more):
    the coarse-fine interfaces lie inside, away from every domain face."""
    from octlb_b200 import Forest, Mesh, TB_WALL, cases
    f = Forest((1, 1, 1), (0, 0, 0), (0, 0, 0, 1, 1, 1)).refine_uniform(2)
    f.refine_box((0.3, 0.3, 0.3, 0.7, 0.7, 0.7), 3)
    if nested:
        f.refine_box((0.45, 0.45, 0.45, 0.55, 0.55, 0.55), 4)
    f.balance().build()
    mesh = Mesh.from_forest(f, 8, tree_boundary_spec=cases._tb_spec(f, lambda b, d: [TB_WALL, 0, 0, 0, -1, 0, 0, 0]))
    assert sorted(set(mesh.levels.tolist())) == ([2, 3, 4] if nested else [2, 3])
    return mesh, np.zeros((mesh.n_blocks, 8, 8, 8, 19))


@pytest.mark.parametrize("nested", [False, True])
def test_const_rho_with_fd_walls_on_several_levels(ob, ref, nested):
    """cavity3d's physics (ConstRhoBGK, the FD walls and lid, the finest
    level's bulk and velocity cells in the statistics) on two and three
    levels: each level's densities carry the shift of its own last collide,
    which the pass removes only where that collide came after the level's
    stream; fields and average_rho against the reference TimeLoop."""
    mesh, init = interior_refined_cavity(ob, nested)
    omega = 1.0 / 0.6
    types = [S.INTERPOLATED_VELOCITY] * 6
    u = np.zeros((6, 3))
    u[3, 0] = 0.05
    lat = ob.GpuLattice(ob.stamp_fd_kinds(mesh, types), omega, init_pops=init)
    lat.set_const_rho(True)
    lat.set_fd_boundary(types, u)
    sim = S(ref, mesh, omega, init)
    sim.set_fd_boundary(types, u, const_rho=True)
    for _ in range(3):
        lat.advance(8)
        sim.advance(8)
        rho_g, u_g = lat.get_fields()
        rho_r, u_r = oracle.rho_u(sim.core())
        eu, er = rel(u_g, u_r), rel(rho_g, rho_r)
        da = abs(lat.average_rho() - sim.average_rho())
        print(f"fd const rho, {3 if nested else 2} levels: u {eu:.2e} rho {er:.2e} average_rho {da:.2e}")
        assert eu <= 1e-5 and er <= 1e-5 and da <= 1e-6
    assert np.abs(u_r).max() > 0.004
    lat.close()


@pytest.mark.parametrize("case", ["cavity3d", "inlet_ramp"])
def test_two_level_mesh(ob, ref, case):
    """The pass on a two-level mesh: after every level step on every level's
    tree-boundary blocks, as the reference's apply_post_stream does, and
    each level's Dirichlet cells collide at that level's next collide (the
    inlet ramp's clock shows it): cavity3d's walls with the moving lid, and a
    box with an inlet on x- ramped over 20 steps against a pressure outlet
    on x+ spanning sixteen blocks."""
    mesh, init = interior_refined_cavity(ob)
    omega = 1.0 / 0.6
    if case == "cavity3d":
        types = [S.INTERPOLATED_VELOCITY] * 6
        u = np.zeros((6, 3))
        u[3, 0] = 0.05
        args = (types, u, np.ones(6), 24, ob.FP32)
        kw = {}
    else:
        types = [S.INTERPOLATED_VELOCITY, S.INTERPOLATED_PRESSURE] + [S.INTERPOLATED_VELOCITY] * 4
        inlet = np.zeros((6, 3))
        inlet[0, 0] = 0.02
        args = (types, np.zeros((6, 3)), np.ones(6), 24, ob.FP32)
        kw = dict(inlet=inlet, ramp=20.0)
    rho_g, u_g, rho_r, u_r = run_pair(ob, ref, mesh, init, omega, *args, **kw)
    print(f"fd two levels {case}: u {rel(u_g, u_r):.2e} rho {rel(rho_g, rho_r):.2e}")
    assert np.abs(u_r).max() > 0.004
    assert rel(u_g, u_r) <= 1e-5 and rel(rho_g, rho_r) <= 1e-5


def test_two_level_mesh_refusals(ob):
    """A coarse-fine interface that meets a domain face (the cavity's band
    under the lid) is refused."""
    from octlb_b200 import cases
    mesh, init, info = cases.cavity_forest(cells=32, n=8, lid=0.0, tau=0.6, band_cells=8)
    types = [S.INTERPOLATED_VELOCITY] * 6
    lat = ob.GpuLattice(ob.stamp_fd_kinds(mesh, types), info["omega"], init_pops=init)
    with pytest.raises(ob.OctlbError) as e:
        lat.set_fd_boundary(types)
    assert e.value.code == ob.capi.OCTLB_EINVAL and "coupler" in str(e.value)
    lat.close()
