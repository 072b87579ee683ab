"""The reference's own domain boundary conditions in the oracle: a
ConcreteDomainBoundaryHandler (Skordos InterpolatedVelocity and pressure
Dirichlet, interpolated_velocity.h:571-1037, domain_boundary_handler.cpp:
60-89) installed in the reference TimeLoop by oracle.Sim.set_fd_boundary.
These CPU tests pin that oracle, and the restatement of the pass in
oracle/fd_boundary.py, which the GPU path is checked against, on properties
of the reconstruction and against the reference's own states:
* a rest state is a fixed point, as in the reference's
  test_interpolated_velocity_compute_rho.cpp equilibrium cases;
* after the post-stream reconstruction every boundary cell carries its
  prescribed velocity, and every plane pressure cell its target density;
* ConstRhoBGK's statistics include the boundary cells."""
import numpy as np
import pytest

from oracle import oracle

S = oracle.Sim


def faces_mask(n):
    m = np.zeros((n, n, n), bool)
    m[0] = m[-1] = True
    m[:, 0] = m[:, -1] = True
    m[:, :, 0] = m[:, :, -1] = True
    return m


def plane_x_max(n):
    m = np.zeros((n, n, n), bool)
    m[-1, 1:-1, 1:-1] = True
    return m


def test_rest_state_is_a_fixed_point(ref):
    """Every face an InterpolatedVelocity wall at rest: the equilibrium at
    rho = 1 stays exactly (the reference's CornerEdge_Equilibrium tests)."""
    from octlb_b200 import cases
    mesh, init, info = cases.cavity_forest(cells=16, n=16, lid=0.0, tau=0.6)
    sim = S(ref, mesh, info["omega"], init)
    sim.set_fd_boundary([S.INTERPOLATED_VELOCITY] * 6)
    sim.advance(10)
    assert np.abs(sim.core()).max() == 0.0


def test_moving_lid_boundary_cells_carry_the_prescribed_velocity(ref):
    """cavity3d's boundary: InterpolatedVelocity on all faces, the lid's
    velocity on the interior top-face cells only (edges and corners of the
    top face stay at rest, interpolated_velocity.h:64-118)."""
    from octlb_b200 import cases
    n = 16
    mesh, init, info = cases.cavity_forest(cells=n, n=n, lid=0.05, tau=0.6)
    u = np.zeros((6, 3))
    u[3, 0] = 0.05
    sim = S(ref, mesh, info["omega"], init)
    sim.set_fd_boundary([S.INTERPOLATED_VELOCITY] * 6, u)
    sim.advance(50)
    rho, vel = oracle.rho_u(sim.core())
    face = faces_mask(n)
    expect = np.zeros((n, n, n, 3))
    expect[1:-1, -1, 1:-1, 0] = 0.05
    assert np.abs(vel[0][face] - expect[face]).max() <= 1e-14
    assert np.abs(vel[0][~face]).max() > 0.01              # the lid drives the cavity
    assert abs(rho[0].mean() - 1.0) < 1e-3                 # the FD walls hold the mass close


def test_pressure_outlet_cells_carry_the_target_density(ref):
    """Lid-driven cavity with a pressure Dirichlet outlet on x+ (rho_target
    1): the outlet's plane cells hold the target density.  Without an inlet
    field the FD path prescribes only the lid's velocity, on the interior
    top-face cells (PrescribedBoundaryU, interpolated_velocity.h:69-117): the
    x- wall's u_wall is not used, so its cells stay at rest."""
    from octlb_b200 import cases
    n = 16
    mesh, init, info = cases.cavity_forest(cells=n, n=n, lid=0.0, tau=0.6)
    types = [S.INTERPOLATED_VELOCITY, S.INTERPOLATED_PRESSURE] + [S.INTERPOLATED_VELOCITY] * 4
    u = np.zeros((6, 3))
    u[0, 0] = 0.02                                          # ignored without an inlet field
    u[3, 0] = 0.05                                          # the lid
    sim = S(ref, mesh, info["omega"], init)
    sim.set_fd_boundary(types, u, rho_target=np.ones(6))
    sim.advance(40)
    rho, vel = oracle.rho_u(sim.core())
    assert np.abs(rho[0][plane_x_max(n)] - 1.0).max() <= 1e-14
    assert np.abs(vel[0][0, 1:-1, 1:-1]).max() <= 1e-14
    assert np.abs(vel[0][1:-1, -1, 1:-1, 0] - 0.05).max() <= 1e-14
    assert np.abs(vel[0][~faces_mask(n)]).max() > 1e-3     # the lid drives the flow


def test_const_rho_statistics_include_the_boundary_cells(ref):
    """With ConstRhoBGK and the FD handler (kFluidAndBoundary statistics,
    time_loop.h:109-115) the average density moves off 1 after a step from a
    compressed state, and the collide holds the mean density near 1."""
    from octlb_b200 import cases, C
    n = 16
    mesh, init, info = cases.cavity_forest(cells=n, n=n, lid=0.05, tau=0.6)
    Cf = C.astype(np.float64)
    w = np.where(np.abs(Cf).sum(1) == 0, 1 / 3, np.where(np.abs(Cf).sum(1) == 1, 1 / 18, 1 / 36))
    init = np.broadcast_to(w * 1.02 - w, init.shape).copy()
    u = np.zeros((6, 3))
    u[3, 0] = 0.05
    sim = S(ref, mesh, info["omega"], init)
    sim.set_fd_boundary([S.INTERPOLATED_VELOCITY] * 6, u, const_rho=True)
    sim.advance(1)
    assert abs(sim.average_rho() - 1.02) < 5e-3
    sim.advance(30)
    rho, _ = oracle.rho_u(sim.core())
    assert abs(rho[0].mean() - 1.0) < 2e-3


def _pass_states(ref, types, u, steps=20):
    from octlb_b200 import cases
    n = 16
    mesh, init, info = cases.cavity_forest(cells=n, n=n, lid=0.0, tau=0.6)
    sim = S(ref, mesh, info["omega"], init)
    sim.set_fd_boundary(types, u, rho_target=np.ones(6))
    sim.advance(steps)
    before, after = sim.advance_phases()
    return before[0], after[0], sim.kinds()[0], info["omega"]


def test_restated_pass_matches_the_reference(ref):
    """oracle/fd_boundary.py (the post-stream reconstruction as plane, edge
    and corner phases, each reading a neighbour's rewritten populations
    exactly when the reference's in-place walk has already rewritten it)
    takes the reference's state after the stream to its state after the
    pass: the moving-lid cavity, and the same with a pressure outlet."""
    from oracle import fd_boundary
    u = np.zeros((6, 3))
    u[3, 0] = 0.05
    for types in ([S.INTERPOLATED_VELOCITY] * 6,
                  [S.INTERPOLATED_VELOCITY, S.INTERPOLATED_PRESSURE] + [S.INTERPOLATED_VELOCITY] * 4):
        before, after, kinds, omega = _pass_states(ref, types, u)
        assert np.abs(after - before).max() > 1e-3            # the pass rewrites the boundary
        got = fd_boundary.reconstruct(before, kinds, omega, u_lid=u[3])
        assert np.abs(got - after).max() <= 1e-14


def test_the_walk_order_matters(ref):
    """Reading every neighbour's original populations instead (no order)
    misses the reference by far more than rounding: edges and corners read
    densities of boundary cells the walk has already rewritten."""
    from oracle import fd_boundary

    class NoOrder(fd_boundary.Block):
        def pops(self, cell, reader):
            return self.f_pre[cell]

    u = np.zeros((6, 3))
    u[3, 0] = 0.05
    before, after, kinds, omega = _pass_states(ref, [S.INTERPOLATED_VELOCITY] * 6, u)
    b = NoOrder(before, kinds, omega, u_lid=u[3])
    cells = [tuple(c) for c in np.argwhere(np.isin(kinds, (fd_boundary.VELOCITY, fd_boundary.PRESSURE)))]
    count = {c: sum(1 for f in b.faces(*c) if f) for c in cells}
    for want, fn in ((1, b.plane), (2, b.edge), (3, b.corner)):
        for c in cells:
            if count[c] == want:
                fn(c)
    got = before.copy()
    for c, f in b.new.items():
        got[c] = f
    assert np.abs(got - after).max() > 1e-4


def test_fd_step_restated_phase_by_phase(ref):
    """A whole step of the reference with the FD conditions, single block
    (halo 1, torus-rotate stream), from its own padded state after each phase
    of TimeLoop::advance_one_with_hooks: the collide (Dirichlet cells at the
    prescribed velocity), no ghost exchange on one block, the linear-rotate
    stream over the padded block (exact, halo included), the post-stream
    padding fill (no change at halo 1) and the reconstruction; composed, the
    restated step gives the reference's state after the step."""
    from octlb_b200 import cases
    from oracle import fd_boundary as fb
    n = 16
    mesh, init, info = cases.cavity_forest(cells=n, n=n, lid=0.0, tau=0.6)
    u = np.zeros((6, 3))
    u[3, 0] = 0.05
    sim = S(ref, mesh, info["omega"], init)
    sim.set_fd_boundary([S.INTERPOLATED_VELOCITY] * 6, u)
    sim.advance(20)
    P = sim.advance_phases_padded()[:, 0]
    kinds = sim.kinds()[0]
    om = info["omega"]
    core = (slice(1, -1),) * 3
    collided = fb.collide(P[0][core], kinds, om, u[3])
    assert np.abs(collided - P[1][core]).max() <= 1e-15
    halo = np.ones((n + 2,) * 3, bool)
    halo[core] = False
    assert np.array_equal(P[1][halo], P[0][halo])          # the halo is not collided
    assert np.array_equal(P[2], P[1])                      # nothing to exchange on one block
    assert np.array_equal(fb.stream_padded(P[2]), P[3])    # exact, halo included
    assert np.array_equal(P[4][halo], P[3][halo])          # the padding fill leaves halo 1 as it is
    assert np.abs(fb.reconstruct(P[3][core], kinds, om, u_lid=u[3]) - P[4][core]).max() <= 1e-14
    # the whole step restated
    p = P[0].copy()
    p[core] = fb.collide(p[core], kinds, om, u[3])
    p = fb.stream_padded(p)
    p[core] = fb.reconstruct(p[core], kinds, om, u_lid=u[3])
    assert np.abs(p - P[4]).max() <= 1e-14


@pytest.mark.parametrize("outlet", [False, True])
def test_restated_pass_matches_the_reference_per_block(ref, outlet):
    """Eight blocks (2 x 2 x 2 level-0 bricks of 8^3): the reference applies
    the reconstruction per block with face, edge and corner roles from the
    block's own extents, so block rims on a domain face are edges and the
    lid moves only on each block's interior top-face cells.  With a pressure
    outlet on x+ (target density 1.002) the outlet spans four blocks: its
    cells on a block rim read u = 0 and density 1 (ExtrapolatedU and
    PrescribedRho off a flat face).  The restatement does the same and
    matches block by block."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_const_rho import brick_cavity
    from oracle import fd_boundary as fb
    mesh, info = brick_cavity(lid=0.0, n=8)
    init = np.zeros((mesh.n_blocks, 8, 8, 8, 19))
    u = np.zeros((6, 3))
    u[3, 0] = 0.05
    types = [S.INTERPOLATED_VELOCITY] * 6
    rho_t = np.ones(6)
    if outlet:
        types[1] = S.INTERPOLATED_PRESSURE
        rho_t[1] = 1.002
    sim = S(ref, mesh, info["omega"], init)
    sim.set_fd_boundary(types, u, rho_target=rho_t)
    sim.advance(15)
    before, after = sim.advance_phases()
    kinds = sim.kinds()
    assert np.abs(after - before).max() > 1e-3
    if outlet:
        assert np.count_nonzero(kinds == fb.PRESSURE) > 0
    for b in range(mesh.n_blocks):
        got = fb.reconstruct(before[b], kinds[b], info["omega"], u_lid=u[3], rho_target=rho_t)
        assert np.abs(got - after[b]).max() <= 1e-14, b


def test_uniform_inlet_with_ramp(ref):
    """A uniform inlet field on x- (UniformInletProfile, inlet_velocity_field.h:
    128-162) and a pressure outlet on x+: every x- cell, edges and corners
    included, carries the ramped inlet velocity (the first face a cell touches
    with an inlet field wins, interpolated_velocity.h:69-102), and the
    restated pass matches the reference.  Steps taken through the hooks keep
    the handler's time at the last advance_one's (19 after 20 steps)."""
    from octlb_b200 import cases
    from oracle import fd_boundary as fb
    n = 16
    mesh, init, info = cases.cavity_forest(cells=n, n=n, lid=0.0, tau=0.6)
    types = [S.INTERPOLATED_VELOCITY, S.INTERPOLATED_PRESSURE] + [S.INTERPOLATED_VELOCITY] * 4
    inlet = np.zeros((6, 3))
    inlet[0, 0] = 0.02
    for ramp_end, t in ((0.0, 0.0), (50.0, 19.0)):
        sim = S(ref, mesh, info["omega"], init)
        sim.set_fd_boundary(types, rho_target=np.ones(6), inlet_u=inlet, ramp_end_t=ramp_end)
        sim.advance(20)
        before, after = sim.advance_phases()
        kinds = sim.kinds()[0]
        got = fb.reconstruct(before[0], kinds, info["omega"], inlets={0: (inlet[0], ramp_end)}, t=t)
        assert np.abs(got - after[0]).max() <= 1e-14
        _, vel = oracle.rho_u(after)
        r = fb.Block.ramp(t, ramp_end)
        assert np.abs(vel[0][0, :, :, 0] - r * 0.02).max() <= 1e-14
        assert (r == 1.0) == (ramp_end == 0.0)


@pytest.mark.parametrize("kind", [2, 3])
def test_poiseuille_inlets_restated(ref, kind):
    """The reference's duct inlet fields on x- of eight 8^3 blocks, ramped
    over 30 steps, against a pressure outlet on x+:
    PoiseuilleInletProfile (kind 2, inlet_velocity_field.h:38-129: the
    parabolas over each block's own in-plane indices, 8 x 8 cells) and
    ChannelPoiseuilleInletProfile (kind 3, :163-269: over the physical
    patch [0.1, 0.9] x [0.2, 0.8] of the face, each block's origin and cell
    width set as cylinder3d sets them).  The restated pass matches the
    reference block by block, and every interior x- cell carries the
    ramped profile."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_const_rho import brick_cavity
    from oracle import fd_boundary as fb
    mesh, info = brick_cavity(lid=0.0, n=8)
    init = np.zeros((mesh.n_blocks, 8, 8, 8, 19))
    types = [S.INTERPOLATED_VELOCITY, S.INTERPOLATED_PRESSURE] + [S.INTERPOLATED_VELOCITY] * 4
    inlet = {"kind": kind, "u": (1.0, 0.0, 0.0), "u_peak": 0.03, "n_inplane": (8, 8),
             "patch": (0.1, 0.9, 0.2, 0.8), "ramp_end_t": 30.0}
    sim = S(ref, mesh, info["omega"], init)
    sim.set_fd_boundary(types, rho_target=np.ones(6), inlets=[inlet, None, None, None, None, None])
    sim.advance(12)
    before, after = sim.advance_phases()
    kinds = sim.kinds()
    t = 11.0
    _, vel = oracle.rho_u(after)
    hit = 0
    for b in range(mesh.n_blocks):
        bd = mesh.bounds[b]
        got = fb.reconstruct(before[b], kinds[b], info["omega"], inlets={0: inlet}, t=t,
                             origin=bd[:3], cell_width=(bd[3] - bd[0]) / 8)
        assert np.abs(got - after[b]).max() <= 1e-14, b
        if bd[0] == 0.0:
            blk = fb.Block(before[b], kinds[b], info["omega"], inlets={0: inlet}, t=t, origin=bd[:3],
                           cell_width=(bd[3] - bd[0]) / 8)
            for y in range(1, 7):
                for z in range(1, 7):
                    want = blk.prescribed_u(0, y, z)
                    assert np.abs(vel[b][0, y, z] - want).max() <= 1e-14
                    hit += want[0] > 0
    assert hit > 0


def test_const_rho_collide_with_fd_conditions_restated(ref):
    """cavity3d's collision: ConstRhoBGK on kBulk cells and the Dirichlet BGK
    on the boundary cells, with the average density from both
    (kFluidAndBoundary): the restated collide gives the reference's state
    after the collide, and the mean of its statistics the reference's next
    average_rho."""
    from octlb_b200 import cases, C
    from oracle import fd_boundary as fb
    n = 16
    mesh, init, info = cases.cavity_forest(cells=n, n=n, lid=0.0, tau=0.6)
    Cf = C.astype(np.float64)
    w = np.where(np.abs(Cf).sum(1) == 0, 1 / 3, np.where(np.abs(Cf).sum(1) == 1, 1 / 18, 1 / 36))
    init = np.broadcast_to(w * 1.01 - w, init.shape).copy()
    u = np.zeros((6, 3))
    u[3, 0] = 0.05
    sim = S(ref, mesh, info["omega"], init)
    sim.set_fd_boundary([S.INTERPOLATED_VELOCITY] * 6, u, const_rho=True)
    sim.advance(7)
    avg = sim.average_rho()
    P = sim.advance_phases_padded()[:, 0]
    kinds = sim.kinds()[0]
    core = (slice(1, -1),) * 3
    stats = []
    got = fb.collide(P[0][core], kinds, info["omega"], u[3], average_rho=avg, stats=stats)
    assert np.abs(got - P[1][core]).max() <= 1e-15
    assert abs(np.mean(stats) - sim.average_rho()) <= 1e-14
    assert abs(avg - 1.0) > 1e-6                             # the correction is active


def test_restated_steps_follow_the_reference_over_time(ref):
    """30 steps of the restated step (collide, linear-rotate stream over the
    padded block, reconstruction) from the reference's padded state stay
    with the reference's own 30 steps: the halo evolves as the reference's,
    so the specification holds over time, not only step by step."""
    from octlb_b200 import cases
    from oracle import fd_boundary as fb
    n = 12
    mesh, init, info = cases.cavity_forest(cells=n, n=n, lid=0.0, tau=0.6)
    u = np.zeros((6, 3))
    u[3, 0] = 0.05
    sim = S(ref, mesh, info["omega"], init)
    sim.set_fd_boundary([S.INTERPOLATED_VELOCITY] * 6, u)
    sim.advance(5)
    P = sim.advance_phases_padded()[:, 0]
    kinds = sim.kinds()[0]
    core = (slice(1, -1),) * 3
    p = P[4].copy()
    for _ in range(30):
        p[core] = fb.collide(p[core], kinds, info["omega"], u[3])
        p = fb.stream_padded(p)
        p[core] = fb.reconstruct(p[core], kinds, info["omega"], u_lid=u[3])
    for _ in range(30):
        q = sim.advance_phases_padded()[4, 0]
    assert np.abs(p - q).max() <= 1e-13
    assert np.abs(q - P[4]).max() > 1e-3                     # the flow moved on
